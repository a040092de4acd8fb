#!/usr/bin/env python
"""Benchmark of the GigaVoxels ray caster on the paged 8192^3 terrain.

Workload (one step = one frame): the seeded fBm terrain voxelised at
8192^3 (2^3-tree of depth 10, 8^3 RGBA8 bricks with a 1-voxel border),
a 2 GiB brick pool in HBM with LRU replacement, 1920x1080 frames along a
256-frame seeded low-altitude camera path.  A frame is the draw (ray cast,
selection mask, histopyramid compaction of the page requests) followed by
the page-request service (de-duplication and classification of the
requests, LRU, brick production and node-word patches, on the GPU).  Rays =
W*H per frame, misses included.  The node pool (322 MB) and brick pool
(2.15 GB) are larger than L2, so no flush is done between frames.

Before timing, paging converges on the path's first frame and the camera
flies the whole path once (untimed); the K timed steps then draw frames
spread evenly over the path (frame k*256/K), so the timed window samples
the whole flight whatever K is.  Besides the headline line's figures the
line carries the ray cast's HBM roofline and instruction-issue fraction,
the checkpointing forward + adjoint, the batched FP16-pool forward of 16
frames in one persistent launch, a full-frame parity check against the
oracles and the CPU baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank renders its own segment of the path (weak scaling,
no collective on the data path).  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s fwd & fwd+bwd, 1080p, 8192³ paged terrain; HBM GB/s vs peak; err vs FP64"
DEPTH, WIDTH, HEIGHT, PATH_FRAMES = 10, 1920, 1080, 256
TERRAIN_SEED, PATH_SEED, JITTER_SEED = 1, 2026, 7
POOL_BYTES = 2 << 30
ALPHA_STOP = 0.99


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=64)
    p.add_argument("--warmup", type=int, default=8)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--workload", default="paged",
                   choices=["paged", "precision", "fit", "batched", "profile-raycast", "profile-adjoint"],
                   help="paged: the 8192^3 paged terrain (default); precision: the 256^3 scene in four brick "
                        "formats against the FP64 oracle; fit: the differentiable 2048^3 variant; batched: 64 "
                        "views of 4 terrains in one persistent launch; profile-raycast / profile-adjoint: a few "
                        "frames of the paged terrain (one renderer, a few GB) for ncu captures")
    p.add_argument("--fit-steps", type=int, default=200)
    p.add_argument("--no-configs", action="store_true",
                   help="skip the config 3/4/5 legs of the default (paged) run")
    p.add_argument("--dump-reference-state", default=None, help=argparse.SUPPRESS)
    return p.parse_args()


def dist_env():
    from voxviz_b200 import dist as vdist

    return vdist.env()


def workload_config(extra=None):
    cfg = {
        "workload": "paged fBm terrain 8192^3 (depth 10, 8^3 RGBA8 bricks + border), 2 GiB LRU brick pool, "
                    "1920x1080, 256-frame seeded low-altitude path; step = draw + page-request service",
        "volume": "8192^3", "depth": DEPTH, "resolution": [WIDTH, HEIGHT], "path_frames": PATH_FRAMES,
        "brick_format": "rgba8", "pool_bytes": POOL_BYTES, "alpha_stop": ALPHA_STOP, "lod": "1 voxel per pixel",
        "seeds": {"terrain": TERRAIN_SEED, "path": PATH_SEED, "jitter": JITTER_SEED},
        "l2": "inputs larger than L2 (node pool 322 MB, brick pool 2.15 GB); no flush",
        "data": "synthetic",
    }
    if extra:
        cfg.update(extra)
    return cfg


class ClockSampler:
    """nvidia-smi samples during the timed region (read-only query)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        """Start sampling every 25 ms and return once the first sample is
        written, so that the sampler is running when the timed region
        starts (nvidia-smi takes a while to come up)."""
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "25"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
            return
        t_end = time.perf_counter() + 5.0
        while time.perf_counter() < t_end and self.p.poll() is None:
            self.f.flush()
            if os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.01)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        rows = [[c.strip() for c in r] for r in rows if r and r[0].strip() == str(self.index)]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# The ray-cast kernel's sources: a profile of the kernel counts only while
# they are unchanged (its summary records their hash).
KERNEL_SOURCES = ("raycast_common.cuh", "kernels.cu", "kernels.cuh", "cellmask.cuh", "lod_bound.h", "fixed_div.h")
ADJOINT_SOURCES = KERNEL_SOURCES + ("adjoint.cu",)


def sources_hash(names) -> str:
    import hashlib

    h = hashlib.sha256()
    for n in names:
        h.update((ROOT / "voxviz_b200" / "csrc" / n).read_bytes())
    return h.hexdigest()[:16]


def ncu_summary(name: str, sources) -> dict | None:
    """Per-launch figures of a kernel from its committed ncu summary
    (profiles/<name>.json), when it was captured on the current sources."""
    p = ROOT / "profiles" / f"{name}.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
    except ValueError:
        return None
    return d if d.get("sources_sha") == sources_hash(sources) else None


def timed_frames(steps: int) -> list[int]:
    """The path frames of the timed steps: spread evenly over the 256-frame
    path whatever the step count, so the timed window always samples the
    whole flight."""
    return [(k * PATH_FRAMES) // steps for k in range(steps)]


def warmup_frames(steps: int, warmup: int) -> list[int]:
    """The warm-up steps: the frames before the first timed one at the same
    spacing."""
    return [((k - warmup) * PATH_FRAMES // steps) % PATH_FRAMES for k in range(warmup)]


def start_renderer(vv, octree, cams, device, steps, warmup, fmt="rgba8", pool_bytes=POOL_BYTES, offset=0):
    """A renderer in the state the timed steps start from: paging converged
    on the path's first frame (cold start), one untimed flight over the whole
    path (frame by frame, every frame drawn and serviced: a pool in steady
    state), then the warm-up steps.  Paging is deterministic, so two calls
    give two renderers in identical states."""
    c = vv.Context(device)
    rr = vv.Renderer(c, octree, fmt=fmt, pool_bytes=pool_bytes, preload_all=False, alpha_stop=ALPHA_STOP,
                     jitter_seed=JITTER_SEED, device_paging=True)
    n_conv = 0
    for n_conv in range(1, 41):
        rr.draw(cams[offset % PATH_FRAMES])
        rr.update()
        if rr.stats()["bricks_uploaded"] == 0:
            break
    for f in range(1, PATH_FRAMES + 1):
        rr.draw(cams[(offset + f) % PATH_FRAMES])
        rr.update()
    for f in warmup_frames(steps, warmup):
        rr.draw(cams[(offset + f) % PATH_FRAMES])
        rr.update()
    return c, rr, n_conv


def cpu_baseline(u_list, words, pool, slots, fmt, jitter, seconds):
    """FP32 oracle on the host cores over whole frames of the same workload
    with the same pools (bounded sample), plus a one-core sample."""
    from oracle import gv_oracle as go

    sc = go.Scene(words, pool, slots, fmt, jitter)
    threads = go.cpu_count()
    rays, t0, frames = 0, time.perf_counter(), 0
    for u in u_list:
        if time.perf_counter() - t0 > seconds:
            break
        go.raycast(u, sc, 32, threads=threads, want_usage=True)
        rays += u.height * u.width
        frames += 1
    dt = time.perf_counter() - t0
    # one core: an eighth of the first frame's rows
    u = u_list[0]
    band = u.height // 8
    t1 = time.perf_counter()
    go.raycast(u, sc, 32, rows=(0, band), threads=1, want_usage=True)
    dt1 = time.perf_counter() - t1
    return {"value": round(rays / dt / 1e6, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"{frames} whole 1920x1080 frames of the timed path, FP32 oracle ray cast with node-usage "
                      f"lists, the GPU's node and brick pools ({rays} rays, {dt:.1f} s)",
            "one_core": {"value": round(band * u.width / dt1 / 1e6, 4), "unit": "Mrays/s", "cores": 1,
                         "sample": f"rows 0-{band} of one frame ({band * u.width} rays, {dt1:.1f} s)"}}


def parity_frame(r, ctx, cam, jitter):
    """The check frame, in full: drawn on the current pools, its node-usage
    lists, selection mask and (after the service) compacted page requests
    compared bit for bit with the FP32 oracle on the pools downloaded before
    the service; its colour against the FP32 oracle, against the FP64 oracle
    (the pixels over 1/255 split into decision flips - the FP64 run takes
    other descent / LOD / step-count / early-termination decisions - and
    pixels with the same decisions whose samples lie elsewhere: binary32
    positions in the normalized volume resolve a voxel of the 8192^3 volume
    to about 1e-3 of its size) and against FP64 arithmetic along the FP32
    sample sequence (arithmetic alone)."""
    from oracle import gv_oracle as go

    r.draw(cam)
    u = r.last_uniforms()
    words = ctx.download_nodes()
    pool = ctx.download_bricks()
    usage, mask = r.read_lists()
    color = r.read_color()
    slots = tuple(int(v) // 10 for v in u.brick_pool_dimension)
    sc = go.Scene(words, pool, slots, ctx.fmt, jitter)
    threads = go.cpu_count()
    c32, u32, st = go.raycast(u, sc, 32, threads=threads)
    m32 = go.select(u32)
    req32, _ = go.compress(u32, m32, 4 * (cam.frame % 3 + 1), u.width * u.height)
    r.update()
    req = r.last_requests()
    flips, c64, _ = go.flip_pixels(u, sc, threads=threads)
    e = np.abs(color.astype(np.float64) - c64)
    px = e.max(axis=-1)
    over = px > 1.0 / 255.0
    ef = np.abs(color.astype(np.float64) - go.fixed_path(u, sc, threads=threads))
    out = {"frame": int(cam.frame), "pixels": int(u.width * u.height),
           "usage_bitexact": bool(np.array_equal(u32, usage)), "mask_bitexact": bool(np.array_equal(m32, mask)),
           "requests_bitexact": bool(np.array_equal(req32, req)), "requests": int(req.shape[0]),
           "colour_max_err_vs_fp32_oracle": float(np.abs(c32 - color).max()), "oracle_status": int(st),
           "err_vs_fp64": {"max": float(e.max()), "rms": float(np.sqrt((e ** 2).mean())),
                           "pixels_over_1_255": float(over.mean())},
           "decision_flip_pixels": float(flips.mean()),
           "over_1_255_decision_flips": float((over & flips).mean()),
           # same decisions, other sample positions: the binary32 positions
           # of the reference's normalized-space arithmetic at 8192^3
           "over_1_255_same_decisions": float((over & ~flips).mean()),
           "err_vs_fp64_same_decisions": {"max": float(px[~flips].max()) if (~flips).any() else 0.0,
                                          "rms": float(np.sqrt((e[~flips] ** 2).mean())) if (~flips).any() else 0.0},
           "err_vs_fp64_same_sample_sequence": {"max": float(ef.max()), "rms": float(np.sqrt((ef ** 2).mean()))}}
    out["bitexact"] = out["usage_bitexact"] and out["mask_bitexact"] and out["requests_bitexact"]
    return out, u, words, pool


# the adjoint's atomics: the timed form and the A/B forms (vv_backward_ex flags)
BWD_MAIN = {"spread": True, "warp_sum": False}
BWD_AB = {"warp_sums": {"spread": False, "warp_sum": True}, "plain": {"spread": False, "warp_sum": False},
          "spread_and_warp_sums": {"spread": True, "warp_sum": True}}


def fwd_bwd_leg(ctx, us, reps, peak, per_ray=16):
    """Checkpointing forward + adjoint of the L2 loss sum(colour^2) over the
    given frames on the current pools.  The texel gradient is sparse: one
    row of 1000 float4 per brick slot the frame touches, claimed by the
    first sample that reaches the slot (vv_backward_ex with a slot map; the
    rows to zero per frame are bounded by the frame's footprint, counted
    before the timed loop).  The timed form spreads the atomics over two
    copies of the rows (VV_GRAD_SPREAD: fewer concurrent atomics on one
    address; the copies are added on the stream, inside the timing); the
    A/B forms (warp sums of the lanes in one cell, VV_GRAD_WARP_SUM; plain
    atomics; both) are timed on the same frames.  Device-timed with CUDA
    events on the stream both run on; the backward's roofline counts its
    algorithmic bytes."""
    import torch

    import voxviz_b200 as vv

    W, H = us[0].width, us[0].height
    dev = torch.device("cuda", torch.cuda.current_device())
    color = torch.empty((H, W, 4), dtype=torch.float32, device=dev)
    nb = vv.Context.ckpt_bytes(W, H, per_ray)
    ck = torch.empty(nb, dtype=torch.uint8, device=dev)
    slots = ctx.slots
    n_slots = slots[0] * slots[1] * slots[2]
    feet = [ctx.footprint(u) for u in us]
    cap = max(b for _, b in feet)
    rows = torch.empty((cap, 1000, 4), dtype=torch.float32, device=dev)
    smap = torch.empty(n_slots, dtype=torch.int32, device=dev)
    used = torch.zeros(1, dtype=torch.int32, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    fwd_ms, bwd_ms, alg_f, alg_b = [], [], [], []
    ab_ms = {name: [] for name in BWD_AB}
    n_ab = min(reps, 8)
    # size the context's copies of the rows for the largest frame (untimed)
    kmax = int(np.argmax([b for _, b in feet]))
    ctx.forward_ckpt(us[kmax], color.data_ptr(), ck.data_ptr(), per_ray)
    smap.fill_(-1)
    used.zero_()
    rows.zero_()
    ctx.backward_ex(us[kmax], color.data_ptr(), ck.data_ptr(), per_ray, rows.data_ptr(), slot_map=smap.data_ptr(),
                    rows_used=used.data_ptr(), rows_cap=cap, spread=True)
    torch.cuda.synchronize()
    runs = [(None, i) for i in range(reps + 2)] + [(name, i) for name in BWD_AB for i in range(n_ab + 1)]
    for mode, i in runs:
        k = i % len(us)
        u = us[k]
        flags = BWD_MAIN if mode is None else BWD_AB[mode]
        ev[0].record()
        ctx.forward_ckpt(u, color.data_ptr(), ck.data_ptr(), per_ray)
        ev[1].record()
        dl = color * 2.0
        smap.fill_(-1)
        used.zero_()
        rows[: feet[k][1]].zero_()
        ctx.backward_ex(u, dl.data_ptr(), ck.data_ptr(), per_ray, rows.data_ptr(), slot_map=smap.data_ptr(),
                        rows_used=used.data_ptr(), rows_cap=feet[k][1], **flags)
        ev[2].record()
        torch.cuda.synchronize()
        if mode is not None:
            if i >= 1:
                ab_ms[mode].append(ev[1].elapsed_time(ev[2]))
        elif i >= 2:
            fwd_ms.append(ev[0].elapsed_time(ev[1]))
            bwd_ms.append(ev[1].elapsed_time(ev[2]))
            n, b = feet[k]
            ckpts = int(ck[: W * H * 8].view(torch.int32).view(H, W, 2)[..., 0].sum())
            reads = 8 * n + (4000 + 128) * b
            # forward: pool reads + colour + checkpoint header and records
            alg_f.append(reads + W * H * (16 + 8) + 48 * ckpts)
            # backward: replay reads + checkpoints + dL/dc + the map and
            # counter + zeroing and read-modify-write of the touched rows
            alg_b.append(reads + W * H * (8 + 16) + 48 * ckpts + 4 * n_slots + 3 * 16000 * int(used.item()))
    status = ctx.device_status(clear=True)
    f, b = float(np.mean(fwd_ms)), float(np.mean(bwd_ms))
    gb_f = float(np.mean(alg_f)) / (f / 1e3) / 1e9
    gb_b = float(np.mean(alg_b)) / (b / 1e3) / 1e9
    return {"fwd_mrays_s": round(W * H / (f / 1e3) / 1e6, 1), "fwd_bwd_mrays_s": round(W * H / ((f + b) / 1e3) / 1e6, 1),
            "fwd_ms": round(f, 3), "bwd_ms": round(b, 3), "frames": len(us), "reps": reps, "per_ray_ckpts": per_ray,
            "ckpt_bytes": nb, "grad_rows_max": cap, "grad_bytes_max": int(cap * 16000),
            "dense_grad_bytes_avoided": int(n_slots * 16000), "status": status,
            "bwd_form": BWD_MAIN,
            "bwd_ms_ab": {name: round(float(np.mean(v)), 3) for name, v in ab_ms.items() if v},
            "roofline": {"forward_ckpt": {"bound": "hbm", "achieved": round(gb_f, 1), "peak": peak, "unit": "GB/s",
                                          "frac": round(gb_f / peak, 4)},
                         "backward": {"bound": "hbm", "achieved": round(gb_b, 1), "peak": peak, "unit": "GB/s",
                                      "frac": round(gb_b / peak, 4),
                                      "formula": "8*nodes + 4128*bricks + W*H*(8 hdr + 16 dL/dc) + 48*checkpoints + "
                                                 "4*slots (map) + 3*16000*rows (zero, read, write)"}},
            "loss": "sum(colour^2); bwd = elementwise dL/dc + slot-map reset + row zeroing + adjoint kernel"}


# 1,040,502 FP16 slots (8000 B each, 102x101x101): near the 102^3 slots 10-bit
# brick pointers address, enough for the 16 views' bricks to converge
def raycast_mode_ab(ctx, us, reps=2):
    """The ray cast of the given frames (on the current pools) launched three
    ways - one thread per pixel in 16x8 tiles; persistent warps that refill
    finished lanes with new pixels; the tiles with each warp's shared brick
    slot staged in shared memory by cp.async.bulk - each launch timed with
    CUDA events (vv_render's profiling events on the context stream); all
    must give the same colour and usage lists."""
    import torch

    import voxviz_b200 as vv

    W, H = us[0].width, us[0].height
    dev = torch.device("cuda", torch.cuda.current_device())
    names = ("tiles", "refill", "staged")
    col = {n: torch.empty((H, W, 4), dtype=torch.float32, device=dev) for n in names}
    use = {n: torch.empty((H, W, 12), dtype=torch.int32, device=dev) for n in names}
    ctx.set_profiling(True)
    ms = {}
    for name in names:
        ctx.set_raycast_mode(name)
        t = []
        for rep in range(reps + 1):
            for u in us:
                ctx.render(u, color=col[name].data_ptr(), usage=use[name].data_ptr(), passes=vv.VV_PASS_RAYCAST)
                a, _ = ctx.last_times()
                if rep:
                    t.append(a)
        ms[name] = float(np.mean(t))
    ctx.set_raycast_mode("tiles")
    same = all(bool(torch.equal(col["tiles"], col[n]) and torch.equal(use["tiles"], use[n])) for n in names[1:])
    ctx.set_profiling(False)
    return {"raycast_ms_tiles": round(ms["tiles"], 4), "raycast_ms_refill": round(ms["refill"], 4),
            "raycast_ms_staged": round(ms["staged"], 4),
            "refill_speedup": round(ms["tiles"] / ms["refill"], 3),
            "staged_speedup": round(ms["tiles"] / ms["staged"], 3), "frames": len(us), "reps": reps,
            "last_frame_bitexact": same}


def compaction_ab(ctx, us, reps=2):
    """The selection + histopyramid + compaction of the given frames (on the
    current pools, after their ray cast) launched both ways - three launches
    (compact.cu) and one launch per pyramid level - each timed with CUDA
    events (vv_render's profiling events); both must give the same mask and
    requests."""
    import torch

    import voxviz_b200 as vv

    W, H = us[0].width, us[0].height
    dev = torch.device("cuda", torch.cuda.current_device())
    use = torch.empty((H, W, 12), dtype=torch.int32, device=dev)
    out = {m: (torch.empty((H, W), dtype=torch.int32, device=dev), torch.empty((W * H, 4), dtype=torch.int32, device=dev),
               torch.zeros(1, dtype=torch.int32, device=dev)) for m in ("three_launch", "per_level")}
    ctx.set_profiling(True)
    ms = {}
    for name in ("three_launch", "per_level"):
        ctx.set_compaction(per_level=name == "per_level")
        mask, req, cnt = out[name]
        t = []
        for rep in range(reps + 1):
            for u in us:
                ctx.render(u, usage=use.data_ptr(), mask=mask.data_ptr(), requests=req.data_ptr(),
                           request_count=cnt.data_ptr(), request_cap=W * H, passes=vv.VV_PASS_ALL)
                _, b = ctx.last_times()
                if rep:
                    t.append(b)
        ms[name] = float(np.mean(t))
    ctx.set_compaction(per_level=False)
    ctx.set_profiling(False)
    a, b = out["three_launch"], out["per_level"]
    n = int(a[2].item())
    same = bool(torch.equal(a[0], b[0]) and n == int(b[2].item()) and torch.equal(a[1][:n], b[1][:n]))
    return {"compact_ms_three_launch": round(ms["three_launch"], 4), "compact_ms_per_level": round(ms["per_level"], 4),
            "frames": len(us), "reps": reps, "last_frame_equal": same}


BATCH16_VIEWS, BATCH16_POOL_BYTES = 16, 8_324_000_000


def batched_fp16_leg(vv, octree, cams, device, peak):
    """The batched FP16-pool forward on the paged 8192^3 terrain: 16 1080p
    frames spread over the path rendered by one persistent launch (autotuned
    tile shape and samples per loop trip) from an 8.3 GB FP16 brick pool
    (1,040,502 slots) with paging run over the 16 views until it converges
    (or for 12 passes), against the same views as per-view launches."""
    import torch

    ctx = vv.Context(device)
    r = vv.Renderer(ctx, octree, fmt="fp16", pool_bytes=BATCH16_POOL_BYTES, preload_all=False,
                    alpha_stop=ALPHA_STOP, jitter_seed=JITTER_SEED, device_paging=True)
    views = [cams[(k * PATH_FRAMES) // BATCH16_VIEWS] for k in range(BATCH16_VIEWS)]
    from voxviz_b200 import scene

    passes, last = scene.converge_views(r, views, 12, strict=False)
    dev = torch.device("cuda", device)
    us = [vv.compute_uniforms(octree.info, cam, ctx.slots, 1.0, ALPHA_STOP) for cam in views]
    bufs = [(torch.empty((u.height, u.width, 4), dtype=torch.float32, device=dev),
             torch.empty((u.height, u.width, 12), dtype=torch.int32, device=dev)) for u in us]
    items = [(ctx, 0, u, c.data_ptr(), q.data_ptr()) for u, (c, q) in zip(us, bufs)]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(reps):
            fn()
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / reps

    def per_view():
        for u, (c, q) in zip(us, bufs):
            ctx.render(u, color=c.data_ptr(), usage=q.data_ptr(), passes=vv.VV_PASS_RAYCAST)

    ms_per_view = timed(per_view)
    ref = [(c.clone(), q.clone()) for c, q in bufs]
    batch = vv.Batch(ctx, items)
    tune = batch.autotune(reps=2)
    ms_batch = timed(batch.render)
    exact = all(bool(torch.equal(a, c)) and bool(torch.equal(b, q)) for (a, b), (c, q) in zip(ref, bufs))
    nodes, bricks = ctx.footprint_union(us)
    rays = sum(u.width * u.height for u in us)
    alg = 8 * nodes + (8000 + 128) * bricks + rays * (16 + 48)
    achieved = alg / (ms_batch / 1e3) / 1e9
    st = r.stats()
    status = ctx.device_status(clear=True)
    out = {"mrays_s": round(rays / (ms_batch / 1e3) / 1e6, 1), "ms": round(ms_batch, 3),
           "per_view_launches_mrays_s": round(rays / (ms_per_view / 1e3) / 1e6, 1),
           "per_view_launches_ms": round(ms_per_view, 3), "views": len(us), "rays": rays,
           "autotune": tune, "bitexact_vs_per_view": exact, "status": status,
           "paging": {"passes": passes, "uploads_in_last_pass": last, "resident": st["resident_bricks"],
                      "pool_slots": st["pool_slots"]},
           "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 4),
                        "algorithmic_bytes": {"per_launch": int(alg), "nodes_touched": int(nodes),
                                              "bricks_touched": int(bricks),
                                              "formula": "8*nodes + (8000 FP16 texels + 128 cell mask)*bricks + "
                                                         "rays*(16 colour + 48 usage), union over the 16 views"}}}
    r.close()
    ctx.close()
    return out


def run_ours(args):
    import torch

    import voxviz_b200 as vv
    from voxviz_b200 import scene

    from voxviz_b200 import dist as vdist

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    vdist.init(timeout_s=600)
    t_setup = time.perf_counter()
    # the octree built on the GPU (heights, mip pyramid, node classification)
    octree = vv.Octree.terrain(seed=TERRAIN_SEED, depth=DEPTH, device=local_rank)
    build_s = time.perf_counter() - t_setup
    heights = octree.heights()
    cams = scene.camera_path(PATH_SEED, heights, PATH_FRAMES, WIDTH, HEIGHT)
    # each rank flies the path from its own starting frame (weak scaling)
    offset, _ = vdist.path_segment(rank, world, PATH_FRAMES)
    frames = [(offset + f) % PATH_FRAMES for f in timed_frames(args.steps)]
    ctx, r, converge = start_renderer(vv, octree, cams, local_rank, args.steps, args.warmup, offset=offset)
    # the end-to-end leg renders the same frames from the same state
    ctx_e, r_e, _ = start_renderer(vv, octree, cams, local_rank, args.steps, args.warmup, offset=offset)
    setup_s = time.perf_counter() - t_setup
    ctx.set_profiling(True)
    vdist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ray_ms, cmp_ms, uploads, requests = [], [], 0, 0
    host_ms = {"ms_readback": 0.0, "ms_visit": 0.0, "ms_policy": 0.0, "ms_produce": 0.0, "ms_upload": 0.0}
    unique_nodes = 0
    timed_u = []
    ev0.record()
    for f in frames:
        r.draw(cams[f])
        r.update()
        a, b = ctx.last_times()
        ray_ms.append(a)
        cmp_ms.append(b)
        st = r.stats()
        uploads += st["bricks_uploaded"]
        requests += st["requests"]
        unique_nodes += st["unique_nodes"]
        for k in host_ms:
            host_ms[k] += st[k]
        timed_u.append(r.last_uniforms())
    ev1.record()
    torch.cuda.synchronize()
    vdist.barrier()
    max_ms = vdist.max_over_ranks(ev0.elapsed_time(ev1), "cuda")
    rays = world * args.steps * WIDTH * HEIGHT
    value = rays / (max_ms / 1e3) / 1e6
    # end to end: same frames through the plugin API with the colour image
    # read back into pinned host memory each step
    # (two pinned buffers, alternating; each frame's copy is queued after its
    # draw and overlaps the page-request service and the next draw; the
    # timed region ends after the last copy has landed)
    hosts = [torch.empty((HEIGHT, WIDTH, 4), dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    vdist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_uploads = 0
    e0.record()
    for k, f in enumerate(frames):
        r_e.draw(cams[f])
        r_e.read_color_async(hosts[k & 1])
        r_e.update()
        e2e_uploads += r_e.stats()["bricks_uploaded"]
    r_e.wait_readback()
    e1.record()
    torch.cuda.synchronize()
    vdist.barrier()
    clk = clocks.stop()  # samples over both timed regions
    e2e_value = rays / (vdist.max_over_ranks(e0.elapsed_time(e1), "cuda") / 1e3) / 1e6
    r_e.close()
    ctx_e.close()
    # roofline of the ray cast: algorithmic bytes of the timed frames (their
    # footprints on the pools at the end of the timed region) over the mean
    # launch duration of the timed region
    ctx.set_profiling(False)
    foot = [ctx.footprint(u) for u in timed_u[:: max(1, len(timed_u) // 8)]]
    nodes = float(np.mean([n for n, _ in foot]))
    bricks = float(np.mean([b for _, b in foot]))
    alg_bytes = 8 * nodes + (4000 + 128) * bricks + WIDTH * HEIGHT * (16 + 48)  # + each slot's cell mask
    peak, peak_kind = measured_peaks()
    ray_mean = float(np.mean(ray_ms))
    achieved = alg_bytes / (ray_mean / 1e3) / 1e9
    prof = ncu_summary("raycast_paged_1080p", KERNEL_SOURCES)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": int(prof["dram_bytes_per_launch"]) if prof else None,
                "kernel": "raycast_kernel<RGBA8>",
                "algorithmic_bytes": {"per_launch": int(alg_bytes), "nodes_touched": int(nodes),
                                      "bricks_touched": int(bricks),
                                      "formula": "8*nodes + (4000 texels + 128 cell mask)*bricks + "
                                                 "W*H*(16 colour + 48 usage); mean over 8 of the timed frames"},
                "traffic_source": prof.get("source") if prof else None}
    if prof:
        # the bound the kernel actually meets: instruction issue, from the
        # captured launch's own instruction count and duration (its frame
        # is not one of the timed frames, so the timed mean is not used)
        n_inst, dur = prof.get("warp_instructions_per_launch"), prof.get("duration_ms_under_ncu")
        roofline["issue"] = {"issue_slots_busy_frac": prof.get("issue_slots_busy_frac"),
                             "warp_instructions_per_launch": n_inst,
                             "captured_launch_ms": dur,
                             "achieved_ginst_s": round(n_inst / (dur / 1e3) / 1e9, 1) if n_inst and dur else None,
                             "peak_ginst_s": round(148 * 4 * (clk.get("sm_mhz") or 1965.0) / 1e3, 1),
                             "note": "one ncu-captured launch (profiles/raycast_paged_1080p.md); peak = 148 SMs x 4 "
                                     "schedulers x 1 warp instruction per clock at the median SM clock of the timed "
                                     "region"}
        if roofline["issue"]["achieved_ginst_s"]:
            roofline["issue"]["frac"] = round(roofline["issue"]["achieved_ginst_s"] /
                                              roofline["issue"]["peak_ginst_s"], 4)
    fb = fwd_bwd_leg(ctx, timed_u[-16:], min(16, args.steps), peak)
    ab = raycast_mode_ab(ctx, timed_u)
    cab = compaction_ab(ctx, timed_u)
    out = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (RGBA8 bricks)", "data": "synthetic",
        "config": workload_config({"parallelism": f"path segments x{world}" if world > 1 else "single GPU"}),
        # per step: camera uniforms, then per uploaded brick one production
        # job (16 B) and about two node-word patches (20 B each: the node and
        # the evicted one); back: the colour image, request count and the
        # distinct node ids (at most 4 per compacted entry)
        "e2e": {"value": round(e2e_value, 2), "unit": "Mrays/s",
                "h2d_bytes_per_step": int(e2e_uploads / args.steps * (16 + 2 * 20) + 256),
                "d2h_bytes_per_step": int(WIDTH * HEIGHT * 16 + 8 + requests / args.steps * 4 * 4)},
        "roofline": roofline,
        "kernels": {"raycast_ms_mean": round(ray_mean, 3),
                    "raycast_ms_min_median_max": [round(float(np.min(ray_ms)), 3), round(float(np.median(ray_ms)), 3),
                                                  round(float(np.max(ray_ms)), 3)],
                    "raycast_mrays_s": round(WIDTH * HEIGHT / (ray_mean / 1e3) / 1e6, 1),
                    "select_compact_ms_mean": round(float(np.mean(cmp_ms)), 3)},
        "paging": {"bricks_uploaded_per_frame": round(uploads / args.steps, 1),
                   "requests_per_frame": round(requests / args.steps, 1), "converge_draws": converge,
                   "distinct_nodes_per_frame": round(unique_nodes / args.steps, 1),
                   "host_ms_per_frame": {k[3:]: round(v / args.steps, 3) for k, v in host_ms.items()},
                   "resident": r.stats()["resident_bricks"], "pool_slots": r.stats()["pool_slots"]},
        "fwd_bwd": fb,
        "raycast_launch_ab": ab,
        "compaction_ab": cab,
        "clocks": clk, "gpu_launches": None, "setup_s": round(setup_s, 1),
        "terrain_build": {"where": "gpu", "seconds": round(build_s, 2)},
    }
    # our kernels per step (as the launch list of profiles/paged_1080p_launch_list.md
    # counts them). draw: raycast + the three-launch selection / histopyramid /
    # compaction; page-request service: request-count read-out, de-duplication
    # (count, first, two scans, scatter), classification (count, scan,
    # scatter), LRU order partition (count, scatter), the candidates'
    # read-out, the pull of jobs and patches, brick production, node patch
    draw_launches = 1 + 3
    service_launches = 1 + 5 + 3 + 2 + 1 + 1 + 1 + 1
    out["gpu_launches"] = args.steps * (draw_launches + service_launches)
    if world == 1:
        out["batched_fp16"] = batched_fp16_leg(vv, octree, cams, local_rank, peak)
    if rank == 0 and not args.no_cpu_baseline:
        jit = vv.make_jitter(JITTER_SEED)
        chk = cams[(frames[-1] + 1) % PATH_FRAMES]
        out["parity"], u_chk, words, pool = parity_frame(r, ctx, chk, jit)
        slots = tuple(int(v) // 10 for v in u_chk.brick_pool_dimension)
        out["cpu_baseline"] = cpu_baseline([u_chk] + timed_u[-12:], words, pool, slots, 0, jit, args.cpu_seconds)
    r.close()
    ctx.close()
    if world == 1 and not args.no_configs:
        # configs 3, 4 and 5 of the workload family in the same run: the
        # brick formats against the FP64 oracle, the batched launch of 64
        # views of 4 terrains, and the differentiable fit (each summarised;
        # `--workload precision|batched|fit` prints them in full)
        sub = argparse.Namespace(**vars(args))
        sub.emit = False
        for key, fn in (("config3_precision", run_precision), ("config4_batched", run_batched),
                        ("config5_fit", run_fit)):
            t0 = time.perf_counter()
            try:
                out[key] = summarise_config(key, fn(sub))
            except Exception as e:  # a failed leg is reported, the headline stands
                out[key] = {"error": f"{type(e).__name__}: {e}"[:300]}
            out[key]["wall_s"] = round(time.perf_counter() - t0, 1)
            torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(out), flush=True)
    vdist.shutdown()


FIT_DEPTH, FIT_VIEWS, FIT_SIZE, FIT_SIGMA, FIT_LR = 8, 16, 512, 0.05, 5e-3
FIT_POOL_BYTES = 6 << 30
FIT_VIEW_SEED, FIT_NOISE_SEED, FIT_FD_SEED = 500, 11, 3


def fit_subvolume_texels(octree, r, grad, slots, n, seed, box=64):
    """`n` random pool texels (slot, texel, channel) with a non-zero gradient
    whose voxel centres lie in a box^3 sub-volume of the leaf-level volume,
    centred on the terrain surface at the volume's centre column."""
    info = octree.info
    L = info.depth
    heights = octree.heights()
    dim = info.volume_dim
    c = np.array([dim // 2, dim // 2, int(heights[dim // 2, dim // 2])])
    lo, hi = c - box // 2, c + box // 2
    xyz, slot = r.residency()
    cand = []
    t = np.arange(1000)
    tl = np.stack([t % 10, (t // 10) % 10, t // 100], axis=1)
    for (x, y, z), s in zip(xyz, slot):
        ni = octree.node_info(int(x), int(y), int(z))
        scale = 1 << (L - ni.level)
        o = np.array(list(ni.origin))
        vox = (o + tl - 1 + 0.5) * scale  # texel centres in leaf voxels (border texels lie outside the node)
        inside = np.all((vox >= lo) & (vox < hi), axis=1) & np.all((tl >= 1) & (tl <= 8), axis=1)
        for ti in np.nonzero(inside)[0]:
            cand.append((int(s), int(ti)))
    if not cand:
        return np.zeros((0, 3), dtype=np.int64), (lo.tolist(), hi.tolist())
    cand = np.array(cand, dtype=np.int64)
    g = grad[cand[:, 0], cand[:, 1]]  # (m, 4)
    nz = np.argwhere(g != 0)
    rng = np.random.default_rng(seed)
    pick = nz[rng.choice(len(nz), size=min(n, len(nz)), replace=False)]
    out = np.stack([cand[pick[:, 0], 0], cand[pick[:, 0], 1], pick[:, 1]], axis=1)
    return out, (lo.tolist(), hi.tolist())


def run_fit(args):
    """Differentiable variant: fit brick contents to target views."""
    import torch

    import voxviz_b200 as vv
    from voxviz_b200 import diff, scene
    from voxviz_b200 import dist as vdist

    # data parallel over views: each rank renders its views, the texel
    # gradient is summed over ranks (the one exchange step), every rank takes
    # the same Adam step
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    vdist.init(timeout_s=900)
    t_setup = time.perf_counter()
    octree = vv.Octree.terrain(seed=TERRAIN_SEED, depth=FIT_DEPTH)
    heights = octree.heights()
    cams = [scene.seeded_view(FIT_VIEW_SEED + v, heights, FIT_SIZE, FIT_SIZE) for v in range(FIT_VIEWS)]
    ctx = vv.Context(local_rank)
    r = vv.Renderer(ctx, octree, fmt="fp32", pool_bytes=FIT_POOL_BYTES, preload_all=False, alpha_stop=ALPHA_STOP,
                    jitter_seed=JITTER_SEED, device_paging=True)
    passes = scene.converge_views(r, cams)
    st = r.stats()
    # keep the z-layers of slots that hold the resident bricks (slots are
    # filled in id order): a smaller pool texture with the same pointers
    sx, sy, _ = ctx.slots
    _, res_slots = r.residency()
    used = int(res_slots.max()) + 1
    slots = (sx, sy, -(-used // (sx * sy)))
    us = [vv.compute_uniforms(octree.info, cam, slots, 1.0, ALPHA_STOP) for cam in cams]
    clean = diff.pool_tensor_from_context(ctx)[: slots[0] * slots[1] * slots[2]].clone()
    diff.attach_pool(ctx, clean, slots)
    torch.cuda.empty_cache()
    gen = torch.Generator(device="cuda").manual_seed(FIT_NOISE_SEED)
    noisy = (clean + FIT_SIGMA * torch.randn(clean.shape, generator=gen, device="cuda")).contiguous()
    with torch.no_grad():
        target = diff.render(noisy, ctx, slots, us)
    del noisy
    setup_s = time.perf_counter() - t_setup
    # the plain ray cast of the same views (no checkpoints), for comparison
    col1 = torch.empty((FIT_SIZE, FIT_SIZE, 4), dtype=torch.float32, device="cuda")
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for rep in range(3):
        if rep == 2:
            p0.record()
        for u in us:
            ctx.render(u, color=col1.data_ptr(), passes=vv.VV_PASS_RAYCAST)
    p1.record()
    torch.cuda.synchronize()
    plain_ms = p0.elapsed_time(p1)
    del col1

    def loss_sum64(c):
        return ((c.double() - target.double()) ** 2).sum()

    # ---- gradient checks at the starting point (param = clean bricks) ----
    param = clean.clone().requires_grad_(True)
    c0 = diff.render(param, ctx, slots, us)
    l0 = loss_sum64(c0)
    l0.backward()
    grad = param.grad.detach()
    status = diff.check_status(ctx)
    gnp = grad.cpu().numpy()
    picks, box = fit_subvolume_texels(octree, r, gnp, slots, 256, FIT_FD_SEED)
    h = 1e-3
    dlc = (2.0 * (c0.detach().double() - target.double())).abs()
    ck1 = torch.empty(vv.Context.ckpt_bytes(FIT_SIZE, FIT_SIZE, 1), dtype=torch.uint8, device="cuda")

    def fd_render(p):
        # colours and per-pixel composited sample counts (checkpoint header)
        # of every view: equal counts = the same control flow
        diff.attach_pool(ctx, p, slots)
        cols = torch.empty((len(us), FIT_SIZE, FIT_SIZE, 4), dtype=torch.float32, device="cuda")
        cnt = []
        for v, u in enumerate(us):
            ctx.forward_ckpt(u, cols[v].data_ptr(), ck1.data_ptr(), 1)
            cnt.append(ck1[: FIT_SIZE * FIT_SIZE * 8].view(torch.int32).view(FIT_SIZE, FIT_SIZE, 2)[..., 1].clone())
        return cols, torch.stack(cnt)

    fd, an, floors, flips = [], [], [], 0
    with torch.no_grad():
        base = param.detach()
        flat = base.view(-1)
        _, n0 = fd_render(base)
        for s_, t_, ch in picks:
            i = (int(s_) * 1000 + int(t_)) * 4 + int(ch)
            old = float(flat[i])
            flat[i] = old + h
            c1, n1 = fd_render(base)
            flat[i] = old - h
            c2, n2 = fd_render(base)
            flat[i] = old
            if not (torch.equal(n1, n0) and torch.equal(n2, n0)):
                flips += 1  # the probe moves a ray across the alpha stop: no derivative there
                continue
            fd.append(float((loss_sum64(c1) - loss_sum64(c2)) / (2 * h)))
            an.append(float(gnp[s_, t_, ch]))
            # binary32 rounding of the two renders on the pixels that changed:
            # each composited sample rounds three times (T, T*src, the sum),
            # so a colour of n samples carries at most (3n+1) u |c|
            steps = (3.0 * n0.double() + 1.0).unsqueeze(-1)
            rnd = 2.0 * steps * torch.maximum(c1.abs(), c2.abs()).double() * 2.0 ** -24
            floors.append(float((dlc * rnd)[c1 != c2].sum()) / (2 * h))
    fd, an, floors = np.array(fd), np.array(an), np.array(floors)
    rel = np.abs(fd - an) / np.maximum(np.abs(an), 1e-30)
    ok = np.abs(fd - an) <= 1e-3 * np.abs(an) + floors
    fd_report = {"texels": int(len(picks)), "h": h, "subvolume_leaf_voxels": box,
                 "control_flow_changes_set_aside": flips, "compared": int(len(fd)),
                 "rel_err_median": float(np.median(rel)) if len(rel) else None,
                 "frac_within_1e-3": float((rel <= 1e-3).mean()) if len(rel) else None,
                 "frac_within_1e-3_plus_fp32_resolution": float(ok.mean()) if len(ok) else None,
                 "criterion": "|fd - grad| <= 1e-3*|grad| + sum over changed pixels of |dL/dc| * 2(3n+1)u|c| / 2h "
                              "(n composited samples, u = 2^-24)",
                 "forward": "binary32 on the GPU", "loss_reduction": "float64 on the GPU"}
    # ---- binary64 host checks on row bands through the sub-volume ----
    # Rays of 16-row bands around the sub-volume centre's projection in every
    # view that sees it: (i) the GPU adjoint against the oracle's binary64
    # adjoint; (ii) central differences of the band loss evaluated in binary64
    # along the binary32 sample sequence (control flow fixed, so the loss is
    # a smooth function of the texels) at 256 random sub-volume texels.
    from oracle import gv_oracle as go
    words = ctx.download_nodes()
    # the resident bricks sit in slots [0, used): only those are read
    _, res_slots = r.residency()
    used = int(res_slots.max()) + 1 if len(res_slots) else 1
    traj_pool = param.detach()[:used].cpu().numpy()
    vals_pool = traj_pool.copy()
    jit = vv.make_jitter(JITTER_SEED)
    osc = go.Scene(words, traj_pool.view(np.uint8).reshape(used, -1), slots, vv.VV_FMT_FP32, jit)
    vsc = go.Scene(words, vals_pool.view(np.uint8).reshape(used, -1), slots, vv.VV_FMT_FP32, jit)
    lo, hi = np.array(box[0], dtype=np.float64), np.array(box[1], dtype=np.float64)
    centre = (lo + hi) / 2.0 / octree.info.volume_dim
    bands = []
    for v, u in enumerate(us):
        C = np.array(list(u.camera_position), dtype=np.float64)
        A = np.stack([np.array(list(u.near_dx)), np.array(list(u.near_dy)), -(centre - C)], axis=1)
        X, Y, a_ = np.linalg.solve(A, -np.array(list(u.near_origin), dtype=np.float64))
        if a_ > 0 and 0 <= X - 0.5 < FIT_SIZE and 0 <= Y - 0.5 < FIT_SIZE:
            yc = int(Y - 0.5)
            r0 = min(max(yc - 8, 0), FIT_SIZE - 16)
            bands.append((v, r0, r0 + 16))
    per_ray = diff.DEFAULT_PER_RAY
    ck = torch.empty(vv.Context.ckpt_bytes(FIT_SIZE, FIT_SIZE, per_ray), dtype=torch.uint8, device="cuda")
    col = torch.empty((FIT_SIZE, FIT_SIZE, 4), dtype=torch.float32, device="cuda")
    # the per-brick gradient reduction of the checks in binary64 on the GPU
    g_gpu = torch.zeros(param.shape, dtype=torch.float64, device="cuda")
    g_ref = np.zeros((used, 1000, 4), dtype=np.float64)
    g_abs = np.zeros((used, 1000, 4), dtype=np.float64)  # magnitude of the summed terms
    dl_np = {}
    for v, r0, r1 in bands:
        ctx.forward_ckpt(us[v], col.data_ptr(), ck.data_ptr(), per_ray)
        dl = torch.zeros_like(col)
        dl[r0:r1] = 2.0 * (col[r0:r1] - target[v, r0:r1])
        ctx.backward_ex(us[v], dl.data_ptr(), ck.data_ptr(), per_ray, g_gpu.data_ptr(), f64=True)
        torch.cuda.synchronize()
        go.backward(us[v], osc, dl.cpu().numpy(), rows=(r0, r1), grad=g_ref, grad_abs=g_abs)
        dl_np[v] = dl[r0:r1].double().cpu().numpy()  # dL/dcolour of the band (held fixed)
    outside = int(torch.count_nonzero(g_gpu[used:]))
    if outside:
        raise RuntimeError(f"{outside} gradient entries outside the resident slots")
    got = g_gpu[:used].cpu().numpy().astype(np.float64)
    scale = float(np.abs(g_ref).max()) if bands else 0.0
    big = np.abs(g_ref) > 1e-3 * scale
    host_rel = (np.abs(got - g_ref)[big] / np.abs(g_ref)[big]) if bands else np.zeros(0)
    nzr = g_ref != 0
    within = np.abs(got - g_ref)[nzr] <= 1e-3 * np.abs(g_ref)[nzr] + 1e-5 * g_abs[nzr]
    host_report = {"bands": [list(b) for b in bands], "rows_per_band": 16, "texels_compared": int(big.sum()),
                   "rel_err_max": float(host_rel.max()) if host_rel.size else None,
                   "abs_err_max_over_max_grad": float(np.abs(got - g_ref).max() / scale) if scale else None,
                   "criterion": "texels above 1e-3 of the largest gradient",
                   "all_texels": int(nzr.sum()),
                   "all_within_1e-3_plus_rounding": float(within.mean()) if within.size else None,
                   "rounding": "1e-5 x the texel's sum of term magnitudes (binary32 per-sample terms)",
                   "gpu_reduction": "binary64"}
    # every resident slot is below `used`, so g_ref covers all candidates
    picks_h, _ = fit_subvolume_texels(octree, r, g_ref, slots, 256, FIT_FD_SEED + 1)
    buf = np.zeros((FIT_SIZE, FIT_SIZE, 4), dtype=np.float64)
    threads = go.cpu_count()

    def band_colours():
        out = []
        for v, r0, r1 in bands:
            go.fixed_path(us[v], osc, vsc, rows=(r0, r1), threads=threads, out=buf)
            out.append(buf[r0:r1].copy())
        return out

    # the functional F = sum(dL/dc * c) over the bands, with dL/dc held at the
    # GPU's value: its texel gradient is exactly what the adjoint returned,
    # and its central difference is taken pixel by pixel (no cancellation)
    flat_vals = vals_pool.reshape(-1)

    def fd_at(i, hh):
        """Central difference of F at flat texel channel i with step hh (as
        stored in binary32)."""
        old = flat_vals[i]
        flat_vals[i] = old + np.float32(hh)
        up_ = float(flat_vals[i])
        c1 = band_colours()
        flat_vals[i] = old - np.float32(hh)
        dn_ = float(flat_vals[i])
        c2 = band_colours()
        flat_vals[i] = old
        return sum(float((dl_np[v] * (a - b)).sum()) for (v, _, _), a, b in zip(bands, c1, c2)) / (up_ - dn_)

    fdh, anh, magh, idx = [], [], [], []
    t_fd = time.perf_counter()
    for s_, t_, ch in picks_h:
        i = (int(s_) * 1000 + int(t_)) * 4 + int(ch)
        idx.append(i)
        fdh.append(fd_at(i, h))
        anh.append(float(got[s_, t_, ch]))
        magh.append(float(g_abs[s_, t_, ch]))
    fdh, anh, magh = np.array(fdh), np.array(anh), np.array(magh)
    relh = np.abs(fdh - anh) / np.maximum(np.abs(fdh), 1e-300)
    okh = np.abs(fdh - anh) <= 1e-3 * np.abs(fdh) + 1e-5 * magh
    # a probe outside the bound: the central difference's own truncation
    # (h^2/6 times the third derivative, for an alpha texel that several
    # samples compound) shows in Richardson's extrapolation from h and h/2,
    # whose truncation is O(h^4)
    richardson = []
    for q in np.nonzero(~okh)[0]:
        f2 = fd_at(idx[q], h / 2)
        rx = (4.0 * f2 - fdh[q]) / 3.0
        richardson.append({"fd_h": float(fdh[q]), "fd_h_2": float(f2), "richardson": float(rx),
                           "gradient": float(anh[q]), "rel_err_h": float(relh[q]),
                           "rel_err_richardson": float(abs(rx - anh[q]) / max(abs(rx), 1e-300)),
                           "channel": int(idx[q] % 4)})
    fd_host_report = {"texels": int(len(picks_h)), "h": h, "evaluation": "binary64 along the binary32 sample sequence",
                      "rel_err_median": float(np.median(relh)) if relh.size else None,
                      "rel_err_max": float(relh.max()) if relh.size else None,
                      "frac_within_1e-3": float((relh <= 1e-3).mean()) if relh.size else None,
                      "frac_within_1e-3_plus_rounding": float(okh.mean()) if relh.size else None,
                      "outside_bound_richardson": richardson,
                      # binary32 per-sample terms that cancel: the error
                      # scaled by max(|fd|, 1e-3 * largest sampled gradient)
                      "scaled_rel_err_max": float((np.abs(fdh - anh) / np.maximum(
                          np.abs(fdh), 1e-3 * np.abs(fdh).max())).max()) if relh.size else None,
                      "seconds": round(time.perf_counter() - t_fd, 1)}
    del traj_pool, vals_pool, got, g_ref, g_abs
    # ---- the fit: Adam on every pool texel, L2 image loss ----
    mine = vdist.views_of_rank(FIT_VIEWS, rank, world)
    us_mine, target_mine = [us[v] for v in mine], target[mine]
    param.grad = None
    opt = torch.optim.Adam([param], lr=FIT_LR, fused=True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    fwd_ms, bwd_ms, adam_ms, losses = [], [], [], []
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for step in range(args.fit_steps):
        ev[0].record()
        c = diff.render(param, ctx, slots, us_mine)
        ev[1].record()
        if world == 1:
            loss = ((c - target) ** 2).mean()
        else:  # this rank's share of the mean over all views
            loss = ((c - target_mine) ** 2).sum() / target.numel()
        opt.zero_grad(set_to_none=True)
        loss.backward()
        vdist.sum_gradients(param.grad)
        ev[2].record()
        opt.step()
        ev[3].record()
        losses.append(loss.detach())
        torch.cuda.synchronize()
        fwd_ms.append(ev[0].elapsed_time(ev[1]))
        bwd_ms.append(ev[1].elapsed_time(ev[2]))
        adam_ms.append(ev[2].elapsed_time(ev[3]))
    t1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = vdist.max_over_ranks(t0.elapsed_time(t1), "cuda")
    # A/B: the same backward with the atomics spread over four copies of the
    # gradient (VV_GRAD_SPREAD, one reduction over the pool after the views)
    spread_bwd_ms = []
    for step in range(4 + 2):
        c = diff.render(param, ctx, slots, us_mine, spread=True)
        loss = ((c - target_mine) ** 2).sum() / target.numel()
        param.grad = None
        ev[1].record()
        loss.backward()
        vdist.sum_gradients(param.grad)
        ev[2].record()
        torch.cuda.synchronize()
        if step >= 2:
            spread_bwd_ms.append(ev[1].elapsed_time(ev[2]))
    param.grad = None
    b_spread = vdist.max_over_ranks(float(np.mean(spread_bwd_ms)), "cuda")
    status |= diff.check_status(ctx)
    if losses:
        lt = torch.stack(losses)
        vdist.sum_gradients(lt)  # the loss over all views
        losses = [float(x) for x in lt.cpu()]
    rays = FIT_VIEWS * FIT_SIZE * FIT_SIZE
    skip = min(3, max(0, args.fit_steps - 1))
    f = vdist.max_over_ranks(float(np.mean(fwd_ms[skip:])), "cuda")
    b = vdist.max_over_ranks(float(np.mean(bwd_ms[skip:])), "cuda")
    a = vdist.max_over_ranks(float(np.mean(adam_ms[skip:])), "cuda")
    out = {
        "workload": "fit", "metric": "Mrays/s fwd & fwd+bwd, 16x512^2 views, 2048^3 FP32 bricks",
        "value": round(rays / ((f + b) / 1e3) / 1e6, 2), "unit": "Mrays/s (fwd+bwd)",
        "fwd_mrays_s": round(rays / (f / 1e3) / 1e6, 2), "higher_is_better": True,
        "plain_raycast_mrays_s": round(rays / (plain_ms / 1e3) / 1e6, 2),
        "ms": {"fwd": round(f, 3), "bwd": round(b, 3), "adam": round(a, 3),
               "step_total_mean": round(total_ms / max(1, args.fit_steps), 3),
               "bwd_with_spread": round(b_spread, 3)},
        "bwd_form": "dense binary32 gradient, plain atomics (A/B: spread over 4 copies, reduced over the pool once "
                    "per step)",
        "adam_steps": args.fit_steps, "lr": FIT_LR,
        "loss": {"first": losses[0] if losses else None, "last": losses[-1] if losses else None,
                 "at": {str(k): losses[k] for k in (0, 10, 50, 100, 199) if k < len(losses)}},
        "grad_check_fd_gpu_fp32": fd_report, "grad_check_fd_fixed_path_fp64": fd_host_report,
        "grad_check_fp64_host_adjoint": host_report, "status": status,
        "config": {"workload": f"fBm terrain {octree.info.volume_dim}^3 (depth {FIT_DEPTH}), FP32 bricks, "
                               f"{FIT_VIEWS} seeded {FIT_SIZE}x{FIT_SIZE} views, targets from bricks + N(0,{FIT_SIGMA})",
                   "pool_slots": list(slots), "resident_bricks": st["resident_bricks"], "paging_passes": passes,
                   "evictions": st["evictions_total"], "params": int(param.numel()), "data": "synthetic",
                   "parallelism": f"views over {world} ranks, texel gradient all-reduced" if world > 1
                   else "single GPU"},
        "n_gpus": world, "clocks": clk, "setup_s": round(setup_s, 1),
    }
    if rank == 0 and getattr(args, "emit", True):
        print(json.dumps(out), flush=True)
    r.close()
    ctx.close()
    vdist.barrier()
    if getattr(args, "emit", True):
        vdist.shutdown()
    return out


BATCH_DEPTHS, BATCH_VIEWS, BATCH_SIDE = (7, 8, 9, 10), 64, (256, 2048)
# per terrain the largest pool 10-bit brick pointers address: 102x101x101
# RGBA8 slots (1,040,502)
BATCH_VIEW_SEED, BATCH_POOL_BYTES, BATCH_PAGING_PASSES = 700, 4_162_008_000, 40


def run_batched(args):
    """Batched variant: 4 terrains (seeds 1..4, depths 7..10), 64 views with
    sides uniform in [256, 2048], paging converged per terrain; per-view
    launches against one persistent launch (autotuned), and a CUDA graph of
    the whole frame (batched ray cast + every view's page-request passes)."""
    import torch

    import voxviz_b200 as vv
    from voxviz_b200 import scene

    torch.cuda.set_device(0)
    t_setup = time.perf_counter()
    rng = np.random.default_rng(BATCH_VIEW_SEED)
    sides = rng.integers(BATCH_SIDE[0], BATCH_SIDE[1] + 1, size=BATCH_VIEWS)
    trees = []
    for k, d in enumerate(BATCH_DEPTHS):
        octree = vv.Octree.terrain(seed=TERRAIN_SEED + k, depth=d)
        ctx = vv.Context(0)
        r = vv.Renderer(ctx, octree, fmt="rgba8", pool_bytes=BATCH_POOL_BYTES, preload_all=False,
                        alpha_stop=ALPHA_STOP, jitter_seed=JITTER_SEED, device_paging=True)
        trees.append({"octree": octree, "ctx": ctx, "r": r, "heights": octree.heights(), "cams": []})
    views = []
    for i in range(BATCH_VIEWS):
        t = trees[i % len(trees)]
        s = int(sides[i])
        cam = scene.seeded_view(BATCH_VIEW_SEED + i, t["heights"], s, s, frame=i)
        t["cams"].append(cam)
        views.append((t, cam))
    # paging state: converged where the pool holds the terrain's 16 views,
    # else the LRU state after BATCH_PAGING_PASSES passes (coarser nodes are
    # drawn where bricks are missing; both launches see the same state)
    passes = [scene.converge_views(t["r"], t["cams"], BATCH_PAGING_PASSES, strict=False) for t in trees]
    dev = torch.device("cuda", 0)
    bufs, items = [], []
    for t, cam in views:
        u = vv.compute_uniforms(t["octree"].info, cam, t["ctx"].slots, 1.0, ALPHA_STOP)
        c = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device=dev)
        us = torch.empty((cam.height, cam.width, 12), dtype=torch.int32, device=dev)
        bufs.append((c, us))
        items.append((t["ctx"], 0, u, c.data_ptr(), us.data_ptr()))
    rays = int(sum(int(cam.width) * int(cam.height) for _, cam in views))
    setup_s = time.perf_counter() - t_setup
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(reps):
            fn()
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / reps

    def per_view():
        for vctx, tree, u, c, us in items:
            vctx.render(u, color=c, usage=us, passes=vv.VV_PASS_RAYCAST, tree=tree)

    ms_per_view = timed(per_view)
    ref = [(c.clone(), us.clone()) for c, us in bufs]
    launch_ctx = trees[0]["ctx"]
    batch = vv.Batch(launch_ctx, items)
    tune = batch.autotune(reps=2)
    ms_batch = timed(batch.render)
    exact = all(bool(torch.equal(a, c)) and bool(torch.equal(b, us)) for (a, b), (c, us) in zip(ref, bufs))
    default_ms = tune["ms"].get("16x16/s1")
    # the frame: batched ray cast + selection / histopyramid / compaction of
    # every view's page requests, eagerly and as one CUDA graph
    req = [(torch.empty((u.height, u.width), dtype=torch.int32, device=dev),
            torch.empty((u.height * u.width, 4), dtype=torch.int32, device=dev),
            torch.zeros(1, dtype=torch.int32, device=dev)) for _, _, u, _, _ in items]

    def frame():
        batch.render()
        for (vctx, tree, u, c, us), (m, rq, cnt) in zip(items, req):
            vctx.render(u, usage=us, mask=m.data_ptr(), requests=rq.data_ptr(), request_count=cnt.data_ptr(),
                        request_cap=u.width * u.height, compress_max_push=4,
                        passes=vv.VV_PASS_SELECT | vv.VV_PASS_COMPACT, tree=tree)

    ms_frame_eager = timed(frame)
    counts_eager = [int(cnt.item()) for _, _, cnt in req]
    # paging in the graph: each terrain's renderer defers its uploads; the
    # host services every view's requests and stages the uploads, the graph
    # applies them (brick production + node patches) before the ray cast
    for t in trees:
        t["r"].set_deferred(True)
        t["r"].stage_uploads()

    def frame_with_uploads():
        for t in trees:
            t["r"].enqueue_uploads()
        frame()

    # the page-request service of a frame: per terrain ONE service of its
    # views' compacted lists concatenated in view order (the distinct nodes in
    # first-seen order over the views, one LRU pass), not one per view
    views_of = [[k for k, (t, _) in enumerate(views) if t is tt] for tt in trees]

    service_parts = {"ms_readback": 0.0, "ms_visit": 0.0, "ms_policy": 0.0, "requests": 0}

    def service_all():
        counts = torch.cat([cnt for _, _, cnt in req]).cpu().tolist()
        for t, ks in zip(trees, views_of):
            lists = [req[k][1][: min(counts[k], items[k][2].width * items[k][2].height)] for k in ks]
            cat = torch.cat(lists) if lists else req[ks[0]][1][:0]
            total = torch.tensor([cat.shape[0]], dtype=torch.int32, device=dev)
            t["r"].service(cat.data_ptr(), total.data_ptr(), max(1, int(cat.shape[0])))
            t["r"].stage_uploads()
            st = t["r"].stats()
            for key in ("ms_readback", "ms_visit", "ms_policy"):
                service_parts[key] += st[key]
            service_parts["requests"] += int(cat.shape[0])

    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for t in trees:
            t["ctx"].set_stream(side.cuda_stream)
        frame_with_uploads()  # sizes every scratch buffer on the capture stream
        side.synchronize()
        with torch.cuda.graph(graph, stream=side):
            frame_with_uploads()
    torch.cuda.synchronize()
    ms_frame_graph = timed(graph.replay)
    counts_graph = [int(cnt.item()) for _, _, cnt in req]
    # whole frames: graph replay, then the host service of all 64 views
    uploads = []
    t0 = time.perf_counter()
    # 3 warm-up frames (the first services after the switch to
    # one service per terrain size their buffers), then 4 timed frames
    warm_frames, paged_frames = 3, 4
    total_before = sum(t["r"].stats()["bricks_uploaded_total"] for t in trees)
    frame_parts = []
    for fi in range(warm_frames + paged_frames):
        if fi == warm_frames:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
        for key in service_parts:
            service_parts[key] = 0
        ta = time.perf_counter()
        graph.replay()
        torch.cuda.synchronize()
        tb = time.perf_counter()
        service_all()
        tc = time.perf_counter()
        total_now = sum(t["r"].stats()["bricks_uploaded_total"] for t in trees)
        uploads.append(int(total_now - total_before))
        total_before = total_now
        frame_parts.append({"warmup": fi < warm_frames,
                            "ms_graph": round((tb - ta) * 1e3, 2), "ms_service": round((tc - tb) * 1e3, 2),
                            **{k: round(v, 2) if k != "requests" else v for k, v in service_parts.items()}})
    torch.cuda.synchronize()
    ms_frame_paged = (time.perf_counter() - t0) / paged_frames * 1e3
    for t in trees:
        t["ctx"].set_stream(0)
    launches_frame = 1 + sum(2 + 2 * (int(np.ceil(np.log2(max(u.width, u.height)))) + 1) for _, _, u, _, _ in items)
    status = max(t["ctx"].device_status() for t in trees)
    out = {
        "workload": "batched", "metric": "Mrays/s, 64 views of 4 paged terrains in one launch",
        "value": round(rays / (ms_batch / 1e3) / 1e6, 1), "unit": "Mrays/s (batched ray cast)",
        "per_view_mrays_s": round(rays / (ms_per_view / 1e3) / 1e6, 1),
        "ms": {"per_view_launches": round(ms_per_view, 3), "batched_autotuned": round(ms_batch, 3),
               "batched_16x16_s1": default_ms, "frame_eager": round(ms_frame_eager, 3),
               "frame_graph_with_staged_uploads": round(ms_frame_graph, 3),
               "frame_graph_plus_host_service": round(ms_frame_paged, 3)},
        "uploads_per_paged_frame": uploads,
        "paged_frame_parts": frame_parts,
        "autotune": tune, "bitexact_vs_per_view": exact,
        "graph_requests_equal_eager": counts_graph == counts_eager,
        "kernel_launches_per_frame": launches_frame, "status": status,
        "config": {"workload": "fBm terrains seeds 1-4 at depths 7/8/9/10 (1024^3..8192^3), RGBA8 bricks, "
                               "4.16 GB LRU pool each (1,040,502 slots), 64 seeded square views with sides uniform "
                               "in [256,2048]; per frame one page-request service per terrain",
                   "rays": rays, "sides": [int(s) for s in sides],
                   "paging": [{"passes": p, "uploads_in_last_pass": u_, "resident": t["r"].stats()["resident_bricks"]}
                              for (p, u_), t in zip(passes, trees)], "data": "synthetic"},
        "setup_s": round(setup_s, 1),
    }
    if getattr(args, "emit", True):
        print(json.dumps(out), flush=True)
    for t in trees:
        t["r"].close()
        t["ctx"].close()
    return out


def run_precision(args):
    """The 256^3 scene in RGBA8 / FP16 / BF16 / FP32 brick pools (and the
    block-compressed DXT5 pool), 64 seeded 512x512 views: Mrays/s, HBM GB/s
    and per-pixel error against the FP64 oracle (on the same stored bricks,
    and on the FP32 bricks)."""
    import torch

    import voxviz_b200 as vv
    from voxviz_b200 import scene
    from oracle import gv_oracle as go

    torch.cuda.set_device(0)
    octree = vv.Octree.terrain(seed=TERRAIN_SEED, depth=5)
    heights = octree.heights()
    jit = vv.make_jitter(JITTER_SEED)
    views = 64
    cams = [scene.seeded_view(3 + v, heights, 512, 512, frame=v) for v in range(views)]
    peak, peak_kind = measured_peaks()
    threads = go.cpu_count()
    ref32 = None
    rows = {}
    order = ["fp32", "rgba8", "fp16", "bf16", "dxt5"]
    for fmt in order:
        f = vv.fmt_code(fmt)
        words, pool, slots, xyz = scene.resident_scene(octree, f)
        ctx = vv.Context(0)
        ctx.upload_nodes(words)
        ctx.create_brickpool(slots, f)
        ctx.upload_bricks(np.arange(xyz.shape[0], dtype=np.uint32), pool[:xyz.shape[0]])
        ctx.set_jitter(jit)
        ctx.set_profiling(True)
        color = torch.empty((512, 512, 4), dtype=torch.float32, device="cuda")
        us = [vv.compute_uniforms(octree.info, c, slots, 1.0, ALPHA_STOP) for c in cams]
        for u in us[:3]:
            ctx.render(u, color=color.data_ptr(), passes=vv.VV_PASS_RAYCAST)
        ms, gbs, imgs = [], [], []
        for u in us:
            ctx.render(u, color=color.data_ptr(), passes=vv.VV_PASS_RAYCAST)
            ctx.synchronize()
            a, _ = ctx.last_times()
            nodes, bricks = ctx.footprint(u)
            ms.append(a)
            gbs.append((8 * nodes + vv.BRICK_BYTES[f] * bricks + 512 * 512 * 16) / (a / 1e3) / 1e9)
            imgs.append(color.cpu().numpy().copy())
        status = ctx.device_status(clear=True)
        sc = go.Scene(words, pool, slots, f, jit)
        own = [go.raycast(u, sc, 64, threads=threads, want_usage=False)[0] for u in us]
        if fmt == "fp32":
            ref32 = own
        e_own = np.concatenate([np.abs(i.astype(np.float64) - o).ravel() for i, o in zip(imgs, own)])
        e_32 = np.concatenate([np.abs(i.astype(np.float64) - o).ravel() for i, o in zip(imgs, ref32)])
        # per pixel: the largest channel error
        px_own = np.concatenate([np.abs(i.astype(np.float64) - o).max(axis=-1).ravel() for i, o in zip(imgs, own)])
        e_fix = np.concatenate([np.abs(i.astype(np.float64) - go.fixed_path(u, sc, threads=threads)).ravel()
                                for i, u in zip(imgs, us)])
        rows[fmt] = {"mrays_s": round(512 * 512 / (float(np.mean(ms)) / 1e3) / 1e6, 1),
                     "raycast_ms": round(float(np.mean(ms)), 4), "hbm_gbs_algorithmic": round(float(np.mean(gbs)), 1),
                     "frac_of_peak": round(float(np.mean(gbs)) / peak, 4),
                     "err_vs_fp64_same_bricks": {"max": float(e_own.max()), "rms": float(np.sqrt((e_own ** 2).mean()))},
                     "err_vs_fp64_fp32_bricks": {"max": float(e_32.max()), "rms": float(np.sqrt((e_32 ** 2).mean()))},
                     "pixels_over_1_255_vs_fp64": float((px_own > 1.0 / 255.0).mean()),
                     "err_vs_fp64_same_sample_sequence": {"max": float(e_fix.max()),
                                                          "rms": float(np.sqrt((e_fix ** 2).mean()))},
                     "status": status, "brick_bytes": vv.BRICK_BYTES[f]}
        ctx.close()
    # the lighting path (GigaVoxels.frag with ComputeLighting): RGBA8 bricks,
    # FP32 gradient bricks, against the FP64 oracle's lit shader
    words, pool, slots, xyz = scene.resident_scene(octree, vv.VV_FMT_RGBA8)
    grads = np.zeros((pool.shape[0], 16000), dtype=np.uint8)
    grads[:xyz.shape[0]] = octree.produce_gradients(xyz, "fp32")
    ctx = vv.Context(0)
    ctx.upload_nodes(words)
    ctx.create_brickpool(slots, "rgba8")
    ctx.upload_bricks(np.arange(xyz.shape[0], dtype=np.uint32), pool[:xyz.shape[0]])
    ctx.create_gradpool("fp32")
    ctx.upload_gradients(np.arange(xyz.shape[0], dtype=np.uint32), grads[:xyz.shape[0]])
    ctx.set_jitter(jit)
    ctx.set_profiling(True)
    color = torch.empty((512, 512, 4), dtype=torch.float32, device="cuda")
    us = [vv.compute_uniforms(octree.info, c, slots, 1.0, ALPHA_STOP) for c in cams]
    for u in us:
        u.compute_lighting = 1
    ms, imgs = [], []
    for u in us[:3]:
        ctx.render(u, color=color.data_ptr(), passes=vv.VV_PASS_RAYCAST)
    for u in us:
        ctx.render(u, color=color.data_ptr(), passes=vv.VV_PASS_RAYCAST)
        ctx.synchronize()
        ms.append(ctx.last_times()[0])
        imgs.append(color.cpu().numpy().copy())
    sc = go.Scene(words, pool, slots, vv.VV_FMT_RGBA8, jit, grads=grads, grad_fmt=vv.VV_FMT_FP32)
    e64 = np.concatenate([np.abs(i.astype(np.float64) - go.raycast(u, sc, 64, threads=threads, want_usage=False)[0])
                          .ravel() for i, u in zip(imgs, us)])
    e32 = max(float(np.abs(i - go.raycast(u, sc, 32, threads=threads, want_usage=False)[0]).max())
              for i, u in zip(imgs[:8], us[:8]))
    rows["rgba8_lit"] = {"mrays_s": round(512 * 512 / (float(np.mean(ms)) / 1e3) / 1e6, 1),
                         "raycast_ms": round(float(np.mean(ms)), 4), "gradients": "fp32",
                         "err_vs_fp32_oracle_max": e32,
                         "err_vs_fp64": {"max": float(e64.max()), "rms": float(np.sqrt((e64 ** 2).mean()))},
                         "status": ctx.device_status(clear=True)}
    ctx.close()
    out = {"workload": "precision", "metric": "Mrays/s, HBM GB/s and error vs FP64 per brick format",
           "config": {"workload": "fBm terrain 256^3 (depth 5), 64 seeded 512x512 views, FP32 compositing",
                      "peak_gbs": peak, "peak_source": peak_kind, "data": "synthetic"},
           "formats": rows, "oracle_threads": threads}
    if getattr(args, "emit", True):
        print(json.dumps(out), flush=True)
    return out


def summarise_config(key, d):
    """The figures of a config run that the headline line carries."""
    if key == "config3_precision":
        return {"formats": {f: {k: v[k] for k in ("mrays_s", "hbm_gbs_algorithmic", "frac_of_peak",
                                                  "err_vs_fp64_same_bricks", "pixels_over_1_255_vs_fp64",
                                                  "err_vs_fp64_same_sample_sequence") if k in v}
                            for f, v in d["formats"].items()}, "config": d["config"]}
    if key == "config4_batched":
        return {k: d[k] for k in ("value", "unit", "per_view_mrays_s", "ms", "bitexact_vs_per_view",
                                  "graph_requests_equal_eager", "uploads_per_paged_frame", "paged_frame_parts",
                                  "autotune", "config")}
    return {k: d[k] for k in ("value", "unit", "fwd_mrays_s", "plain_raycast_mrays_s", "ms", "bwd_form", "adam_steps",
                              "loss",
                              "grad_check_fd_gpu_fp32", "grad_check_fd_fixed_path_fp64",
                              "grad_check_fp64_host_adjoint", "status", "config")}


def run_profile(args):
    """A small case of the paged workload for ncu captures (one renderer, a
    few GB on the device): paging converged on the path's first frame, then
    frames 1..3 drawn and serviced.  profile-adjoint then runs the
    checkpointing forward and the adjoint of frame 3 (sparse gradient).
    Prints the kernel launch counts so a capture can skip to a chosen launch."""
    import torch

    import voxviz_b200 as vv
    from voxviz_b200 import scene

    torch.cuda.set_device(0)
    octree = vv.Octree.terrain(seed=TERRAIN_SEED, depth=DEPTH)
    cams = scene.camera_path(PATH_SEED, octree.heights(), PATH_FRAMES, WIDTH, HEIGHT)
    ctx = vv.Context(0)
    r = vv.Renderer(ctx, octree, fmt="rgba8", pool_bytes=POOL_BYTES, preload_all=False, alpha_stop=ALPHA_STOP,
                    jitter_seed=JITTER_SEED, device_paging=True)
    draws = 0
    for _ in range(40):
        r.draw(cams[0])
        r.update()
        draws += 1
        if r.stats()["bricks_uploaded"] == 0:
            break
    for f in (1, 2, 3):
        r.draw(cams[f])
        r.update()
        draws += 1
    out = {"workload": args.workload, "raycast_launches": draws}
    if args.workload == "profile-adjoint":
        fb = fwd_bwd_leg(ctx, [r.last_uniforms()], 1, measured_peaks()[0])
        out["fwd_bwd"] = fb
    torch.cuda.synchronize()
    out["status"] = ctx.device_status()
    print(json.dumps(out), flush=True)
    r.close()
    ctx.close()


def dump_reference_state(args):
    """Set-up step of the reference arm, run in its own process: the GPU arm's
    state at the start of its timed window (node words, brick pool, LRU order
    and residency after the cold start, the untimed flight and the warm-up
    steps), the uniforms of the timed frames, and the brick store the timed
    steps page in (every brick they upload, as the reference's pager reads
    bricks from its store), written as .npy files for a process that never
    loads the CUDA library."""
    import voxviz_b200 as vv
    from voxviz_b200 import scene

    out = Path(args.dump_reference_state)
    out.mkdir(parents=True, exist_ok=True)
    octree = vv.Octree.terrain(seed=TERRAIN_SEED, depth=DEPTH)
    cams = scene.camera_path(PATH_SEED, octree.heights(), PATH_FRAMES, WIDTH, HEIGHT)
    ctx, r, _ = start_renderer(vv, octree, cams, 0, args.steps, args.warmup)
    np.save(out / "words.npy", ctx.download_nodes())
    np.save(out / "pool.npy", ctx.download_bricks())
    np.save(out / "lru.npy", r.lru_order())
    xyz, slot = r.residency()
    np.save(out / "res_xyz.npy", xyz)
    np.save(out / "res_slot.npy", slot)
    np.save(out / "jitter.npy", vv.make_jitter(JITTER_SEED))
    frames = timed_frames(args.steps)
    us = []
    # every node the window pages in: the paging policy run on the GPU's
    # requests gives each step's uploads (the GPU's residency equals it)
    from oracle.paging_ref import PagingRef

    sim = PagingRef(ctx.download_nodes(), tuple(ctx.slots))
    sim.set_state(r.lru_order(), xyz, slot)
    paged = set()
    for f in frames:
        r.draw(cams[f])
        r.update()
        us.append(bytes(r.last_uniforms()))
        paged.update(sim.update(r.last_requests()))
    xyz2, slot2 = r.residency()
    if {tuple(int(v) for v in p): int(s) for p, s in zip(xyz2, slot2)} != sim.residency():
        raise RuntimeError("the paging policy and the GPU service disagree")
    paged = np.array(sorted(paged) or [(0, 0, 0)], dtype=np.uint32)
    np.save(out / "uniforms.npy", np.frombuffer(b"".join(us), dtype=np.uint8).reshape(len(us), -1))
    np.save(out / "end_xyz.npy", xyz2)
    np.save(out / "end_slot.npy", slot2)
    np.save(out / "end_lru.npy", r.lru_order())
    st = r.stats()
    np.save(out / "store_xyz.npy", paged)
    np.save(out / "store_bricks.npy", octree.produce_bricks(paged, "rgba8"))
    (out / "meta.json").write_text(json.dumps({"frames": frames, "evictions_total": st["evictions_total"],
                                               "slots": list(ctx.slots)}))
    r.close()
    ctx.close()


def run_reference(args):
    """The reference's algorithm on the host cores (its GLSL path needs a
    graphics stack, unavailable on this box): the FP32 oracle port of
    GigaVoxelsNoLighting.frag and of the compaction passes
    (GenerateSelectionMask / ComputeActiveTexels / GenerateHistoPyramid /
    CompressNodeUsageList), then the page-request service
    (NodeUsageListProcessor::run + BrickPool::update restated in
    oracle/paging_ref.py, bricks copied in from the brick store), on the same
    frames from the same paging state as the GPU arm, all host cores.  The
    state comes from a set-up process; this process never loads the CUDA
    library."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    import shutil

    from oracle import gv_oracle as go
    from oracle.paging_ref import PagingRef
    from voxviz_b200._native import Uniforms

    go.build()
    tmp = Path(tempfile.mkdtemp(prefix="vv_refstate_"))
    try:
        t_setup = time.perf_counter()
        cmd = [sys.executable, str(ROOT / "bench.py"), "--dump-reference-state", str(tmp), "--steps", str(args.steps),
               "--warmup", str(args.warmup)]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            print(json.dumps({"impl": "reference", "unavailable": "set-up process failed: " +
                              (p.stderr.strip().splitlines() or ["?"])[-1][:200]}), flush=True)
            return
        meta = json.loads((tmp / "meta.json").read_text())
        slots = tuple(meta["slots"])
        words = np.load(tmp / "words.npy")
        pool = np.load(tmp / "pool.npy")
        sim = PagingRef(words, slots)
        sim.set_state(np.load(tmp / "lru.npy"), np.load(tmp / "res_xyz.npy"), np.load(tmp / "res_slot.npy"))
        ub = np.load(tmp / "uniforms.npy")
        us = [Uniforms.from_buffer_copy(ub[i].tobytes()) for i in range(ub.shape[0])]
        store_xyz = np.load(tmp / "store_xyz.npy")
        store_bricks = np.load(tmp / "store_bricks.npy")
        store = {tuple(int(v) for v in xyz): i for i, xyz in enumerate(store_xyz)}
        jit = np.load(tmp / "jitter.npy")
        sc = go.Scene(sim.words, pool, slots, 0, jit)
        threads = go.cpu_count()
        setup_s = time.perf_counter() - t_setup
        # warm-up: draws of the first timed frame (no service: the state stays)
        for _ in range(min(args.warmup, 2)):
            go.raycast(us[0], sc, 32, threads=threads)
        missing = 0
        t0 = time.perf_counter()
        for k, u in enumerate(us):
            _, usage, _ = go.raycast(u, sc, 32, threads=threads)
            mask = go.select(usage)
            # CompressNodeUsageList's MaxNodesToPush of the frame: 4 * (frame % 3 + 1)
            req, _ = go.compress(usage, mask, 4 * (meta["frames"][k] % 3 + 1), u.width * u.height)
            for n in sim.update(req):
                i = store.get(n)
                s_ = sim.node_slot[n]
                if i is None:
                    missing += 1
                else:
                    pool[s_] = store_bricks[i]
        dt = time.perf_counter() - t0
        # the paging state both arms reach at the end of the window
        end_res = {tuple(int(v) for v in p): int(s) for p, s in zip(np.load(tmp / "end_xyz.npy"),
                                                                      np.load(tmp / "end_slot.npy"))}
        same_state = end_res == sim.residency() and bool(np.array_equal(np.load(tmp / "end_lru.npy"),
                                                                        sim.lru_order()))
        # one core: an eighth of the first timed frame's rows
        band = HEIGHT // 8
        t1 = time.perf_counter()
        go.raycast(us[0], sc, 32, rows=(0, band), threads=1)
        dt1 = time.perf_counter() - t1
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    loaded = any("libvoxviz_b200" in line for line in Path("/proc/self/maps").read_text().splitlines())
    rays = len(us) * WIDTH * HEIGHT
    value = rays / dt / 1e6
    out = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (RGBA8 bricks)",
        "data": "synthetic",
        "config": workload_config({"parallelism": "single GPU"}),
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
                         "sample": f"the {args.steps} timed steps in full: 1920x1080 FP32 oracle ray cast, selection "
                                   f"mask, histopyramid compaction and the page-request service, from the GPU "
                                   f"arm's paging state",
                         "one_core": {"value": round(band * WIDTH / dt1 / 1e6, 4), "unit": "Mrays/s", "cores": 1,
                                      "sample": f"rows 0-{band} of the first timed frame"}},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "same_paging_state_at_end": same_state, "bricks_missing_from_store": missing,
        "product_library_loaded": loaded, "setup_s": round(setup_s, 1),
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.dump_reference_state:
        dump_reference_state(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "fit":
        run_fit(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "precision":
        run_precision(args)
    elif args.workload.startswith("profile-"):
        run_profile(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
