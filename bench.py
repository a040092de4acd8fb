#!/usr/bin/env python
"""Benchmark of the GigaVoxels ray caster on the paged 8192^3 terrain.

Workload (one step = one frame): the seeded fBm terrain voxelised at
8192^3 (2^3-tree of depth 10, 8^3 RGBA8 bricks with a 1-voxel border),
a 2 GiB brick pool in HBM with LRU replacement, 1920x1080 frames along a
256-frame seeded low-altitude camera path.  A frame is the draw (ray cast,
selection mask, histopyramid compaction of the page requests) followed by
the page-request service (request read-back, LRU, brick production on the
host cores, upload, node-word patches).  Rays = W*H per frame, misses
included.  The node pool (322 MB) and brick pool (2.15 GB) are larger
than L2, so no flush is done between frames.

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
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


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
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

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


RAYCAST_VERSION = "v2"  # bumped whenever the ray-cast kernel changes; the ncu capture must match


def ncu_traffic():
    """Per-launch DRAM bytes of the ray cast from the committed ncu summary,
    when it was captured on the current kernel version."""
    p = ROOT / "profiles" / "raycast_paged_1080p_traffic.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
        except ValueError:
            return None
        return d if d.get("kernel_version") == RAYCAST_VERSION else None
    return None


def cpu_baseline(u_list, words, pool, slots, fmt, jitter, seconds):
    """FP32 oracle on the host cores over the same frames (bounded sample)."""
    from oracle import gv_oracle as go

    sc = go.Scene(words, pool, slots, fmt, jitter)
    threads = go.cpu_count()
    rays, t0, frames = 0, time.perf_counter(), 0
    H = u_list[0].height
    band = max(1, H // 8)
    i = 0
    while time.perf_counter() - t0 < seconds and i < 8 * len(u_list):
        u = u_list[i % len(u_list)]
        r0 = (i * band) % H
        r1 = min(H, r0 + band)
        go.raycast(u, sc, 32, rows=(r0, r1), threads=threads, want_usage=True)
        rays += (r1 - r0) * u.width
        frames += 1
        i += 1
    dt = time.perf_counter() - t0
    return {"value": rays / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"{frames} row bands of 1/8 frame (1920x{band}) from the timed frames, FP32 oracle, "
                      f"same node/brick pools as the GPU ({rays} rays, {dt:.1f} s)"}


def parity_sample(r, ctx, u, words, pool, slots, fmt, jitter):
    """GPU frame vs the FP32 oracle (bit-exact lists) and the FP64 oracle (error) on row bands."""
    from oracle import gv_oracle as go

    usage, mask = r.read_lists()
    color = r.read_color()
    sc = go.Scene(words, pool, slots, fmt, jitter)
    bands = [(y, y + 8) for y in range(0, u.height, u.height // 6)][:6]
    exact, err_max, sq, n = True, 0.0, 0.0, 0
    for r0, r1 in bands:
        r1 = min(r1, u.height)
        c32, u32, _ = go.raycast(u, sc, 32, rows=(r0, r1))
        c64, _, _ = go.raycast(u, sc, 64, rows=(r0, r1), want_usage=False)
        exact &= bool(np.array_equal(u32[r0:r1], usage[r0:r1]))
        exact &= bool(np.abs(c32[r0:r1] - color[r0:r1]).max() <= 1.0 / 255.0)
        e = np.abs(color[r0:r1].astype(np.float64) - c64[r0:r1])
        err_max = max(err_max, float(e.max()))
        sq += float((e ** 2).sum())
        n += e.size
    return {"rows_checked": sum(b - a for a, b in bands), "usage_bitexact_vs_fp32_oracle": exact,
            "err_vs_fp64": {"max": err_max, "rms": (sq / max(n, 1)) ** 0.5}}


def run_ours(args):
    import torch

    import voxviz_b200 as vv
    from voxviz_b200 import scene

    rank, local_rank, world = dist_env()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local_rank)
    t_setup = time.perf_counter()
    octree = vv.Octree.terrain(seed=TERRAIN_SEED, depth=DEPTH)
    heights = octree.heights()
    cams = scene.camera_path(PATH_SEED, heights, PATH_FRAMES, WIDTH, HEIGHT)
    offset = rank * PATH_FRAMES // world

    def start_renderer():
        """A renderer in the state the timed frames start from: paging
        converged on the segment's first frame (cold start), then the
        warm-up frames.  Paging is deterministic, so two calls give two
        renderers in identical states."""
        c = vv.Context(local_rank)
        rr = vv.Renderer(c, octree, fmt="rgba8", pool_bytes=POOL_BYTES, preload_all=False, alpha_stop=ALPHA_STOP,
                         jitter_seed=JITTER_SEED, device_paging=True)
        n_conv = 0
        for n_conv in range(1, 41):
            rr.draw(cams[offset])
            rr.update()
            if rr.stats()["bricks_uploaded"] == 0:
                break
        f = offset + 1
        for _ in range(args.warmup):
            rr.draw(cams[f % PATH_FRAMES])
            rr.update()
            f += 1
        return c, rr, n_conv, f

    ctx, r, converge, frame = start_renderer()
    # the end-to-end leg renders the same frames from the same state
    ctx_e, r_e, _, frame_e = start_renderer()
    setup_s = time.perf_counter() - t_setup
    ctx.set_profiling(True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ray_ms, cmp_ms, uploads, requests = [], [], 0, 0
    host_ms = {"ms_readback": 0.0, "ms_policy": 0.0, "ms_produce": 0.0, "ms_upload": 0.0}
    timed_u = []
    ev0.record()
    for _ in range(args.steps):
        r.draw(cams[frame % PATH_FRAMES])
        r.update()
        a, b = ctx.last_times()
        ray_ms.append(a)
        cmp_ms.append(b)
        st = r.stats()
        uploads += st["bricks_uploaded"]
        requests += st["requests"]
        for k in host_ms:
            host_ms[k] += st[k]
        timed_u.append(r.last_uniforms())
        frame += 1
    ev1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    elapsed = ev0.elapsed_time(ev1)
    t = torch.tensor([elapsed], device="cuda")
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    rays = world * args.steps * WIDTH * HEIGHT
    value = rays / (max_ms / 1e3) / 1e6
    # end to end: same frames through the plugin API with the colour image
    # read back into pinned host memory each step
    host = torch.empty((HEIGHT, WIDTH, 4), dtype=torch.float32, pin_memory=True)
    host_np = host.numpy()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_uploads = 0
    e0.record()
    for _ in range(args.steps):
        r_e.draw(cams[frame_e % PATH_FRAMES])
        r_e.update()
        r_e.read_color(host_np)
        e2e_uploads += r_e.stats()["bricks_uploaded"]
        frame_e += 1
    e1.record()
    torch.cuda.synchronize()
    te = torch.tensor([e0.elapsed_time(e1)], device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = rays / (float(te.item()) / 1e3) / 1e6
    # check frame: the next frame of the path drawn on the current pools (no
    # update after it), so the downloaded pools are exactly what it read
    r.draw(cams[frame % PATH_FRAMES])
    chk_ray_ms, _ = ctx.last_times()
    ctx.set_profiling(False)
    u_last = r.last_uniforms()
    # roofline of the ray cast: algorithmic bytes of the check frame (same
    # path, same pools) over the mean launch duration of the timed region
    nodes, bricks = ctx.footprint(u_last)
    alg_bytes = 8 * nodes + 4000 * bricks + WIDTH * HEIGHT * (16 + 48)
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (float(np.mean(ray_ms)) / 1e3) / 1e9
    traffic = ncu_traffic()
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
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "traffic": traffic.get("bytes_per_launch") if traffic else None,
                     "kernel": "raycast_kernel<RGBA8>",
                     "algorithmic_bytes": {"per_launch": int(alg_bytes), "nodes_touched": int(nodes),
                                           "bricks_touched": int(bricks),
                                           "formula": "8*nodes + 4000*bricks + W*H*(16 colour + 48 usage)",
                                           "measured_on": "check frame after the timed region",
                                           "check_frame_raycast_ms": round(chk_ray_ms, 3)},
                     "traffic_source": (traffic or {}).get("source")},
        "kernels": {"raycast_ms_mean": round(float(np.mean(ray_ms)), 3),
                    "raycast_mrays_s": round(WIDTH * HEIGHT / (np.mean(ray_ms) / 1e3) / 1e6, 1),
                    "select_compact_ms_mean": round(float(np.mean(cmp_ms)), 3)},
        "paging": {"bricks_uploaded_per_frame": round(uploads / args.steps, 1),
                   "requests_per_frame": round(requests / args.steps, 1), "converge_draws": converge,
                   "host_ms_per_frame": {k[3:]: round(v / args.steps, 3) for k, v in host_ms.items()},
                   "resident": r.stats()["resident_bricks"], "pool_slots": r.stats()["pool_slots"]},
        "clocks": clk, "gpu_launches": None, "setup_s": round(setup_s, 1),
    }
    # our kernels per step: raycast + select + (levels-1) up + (levels-1) down + total + compact + patch + scatter
    levels = 11
    out["gpu_launches"] = args.steps * (1 + 1 + 2 * (levels - 1) + 1 + 1) + 2 * args.steps
    if rank == 0 and not args.no_cpu_baseline:
        words = ctx.download_nodes()
        pool = ctx.download_bricks()
        jit = vv.make_jitter(JITTER_SEED)
        slots = tuple(int(v) // 10 for v in u_last.brick_pool_dimension)
        out["parity"] = parity_sample(r, ctx, u_last, words, pool, slots, 0, jit)
        out["cpu_baseline"] = cpu_baseline([u_last] + timed_u[-3:], words, pool, slots, 0, jit, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(out), flush=True)
    r.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def run_reference(args):
    """The reference's algorithm on the host cores: the FP32 oracle port (the
    reference's own GLSL path cannot run here: no graphics stack)."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    import voxviz_b200 as vv
    from voxviz_b200 import scene
    from oracle import gv_oracle as go
    from oracle.host_scene import HostScene

    go.build()
    octree = vv.Octree.terrain(seed=TERRAIN_SEED, depth=DEPTH)
    cams = scene.camera_path(PATH_SEED, octree.heights(), PATH_FRAMES, WIDTH, HEIGHT)
    slots = scene.slot_grid(POOL_BYTES // 4000)
    jit = vv.make_jitter(JITTER_SEED)
    hs = HostScene(octree, slots, 0, jit)
    threads = go.cpu_count()
    band = HEIGHT // 16
    frames = [1 + k for k in range(args.warmup + args.steps)]
    us = [vv.compute_uniforms(octree.info, cams[f % PATH_FRAMES], slots, 1.0, ALPHA_STOP) for f in frames]
    rows = [((k * 7 * band) % (HEIGHT - band), (k * 7 * band) % (HEIGHT - band) + band) for k in range(len(frames))]
    # make the sampled rays' bricks resident (the converged paging state), untimed
    for u, rr in zip(us, rows):
        hs.converge([u], rows=rr, threads=threads)
    for k in range(args.warmup):
        go.raycast(us[k], hs.scene, 32, rows=rows[k], threads=threads)
    t0 = time.perf_counter()
    rays = 0
    for k in range(args.warmup, len(frames)):
        go.raycast(us[k], hs.scene, 32, rows=rows[k], threads=threads)
        rays += (rows[k][1] - rows[k][0]) * WIDTH
    dt = time.perf_counter() - t0
    value = rays / dt / 1e6
    out = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config({"reference_sample": f"1/16 of each frame's rows (1920x{band}), one band per step"}),
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} steps x 1920x{band} rays, bricks made resident on the host "
                                   f"first ({hs.next_slot} bricks)"},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
