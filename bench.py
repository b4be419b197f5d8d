#!/usr/bin/env python
"""Benchmark of the GPU visibility path (meshlets culled per second).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step is one pass of the hot path over one synthetic frame: Hi-Z pyramid build
from the frame's depth, object LOD select, meshlet cull and deterministic draw
compaction, for every view of the workload. The metric counts (view, LOD0 scene
meshlet) pairs per second. Inputs are resident in HBM for `value`; `e2e` runs
the same step through the C-ABI with host buffers (depth and camera copied in,
counters and visible draws copied out) inside the timed region.

Workloads: plain2 (default; 100,000 instances x 100 meshlets = 10M LOD0 meshlets,
3840x2160, one view), plain1 (1M meshlets, 1920x1080), plain0 (262,144 meshlets,
1024x1024).

Multi-GPU (torchrun): every rank runs its own replica of the workload on its own
GPU (independent frames, no collective on the data path): weak scaling, time =
max over ranks. `--impl reference` times the CPU restatement of the reference
shaders (the oracle) on the host cores, on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="plain2", choices=["plain2", "plain1", "plain0"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="bound of the CPU baseline sample")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def build_workload(name: str):
    from helio_b200 import scene as S

    cfg = {"plain2": 2, "plain1": 1, "plain0": 0}[name]
    return S.config(cfg)


def hiz_bytes(w: int, h: int, copy: bool) -> int:
    b = 4 * w * h * (2 if copy else 1)
    m = min(int(max(w, h)).bit_length(), 12)
    for l in range(1, m):
        b += 4 * max(w >> l, 1) * max(h >> l, 1)
    return b


def vg_algorithmic_bytes(scene, selected: np.ndarray, visible: int) -> dict:
    """Bytes an ideal implementation must move per launch, from the step's own outputs.
    select: per object 64 B (head, local bounds, LOD errors) + 64 B model + 16 B
    InstanceCullData + 4 B selected-LOD write + 16 B selected range record.
    cull: per work item 8 B item + 8 B selected range + 8 B visibility bitmask; per
    active work item 80 B (model + cull data); per tested meshlet 44 B (centre, radius,
    cone apex, cutoff, axis as f32); per visible meshlet 12 B read + 20 B + 16 B written."""
    obj = scene.objects
    items = scene.work_items
    O, W = len(obj), len(items)
    sp1 = selected.astype(np.int64)
    lod = np.maximum(sp1 - 1, 0)
    cnt = np.where(sp1 > 0, obj["lod_meshlet_counts"][np.arange(O), lod], 0)
    oi = items["object_index"].astype(np.int64)
    valid = oi < O
    c = np.zeros(W, np.int64)
    c[valid] = cnt[oi[valid]]
    base = items["local_meshlet_base"].astype(np.int64)
    n = np.clip(c - base, 0, 64)
    tested = int(n.sum())
    active = int((n > 0).sum())
    return {"select": 164 * O, "cull_test": 24 * W + 80 * active + 44 * tested, "cull_emit": 48 * visible,
            "tested_meshlets": tested, "active_items": active}


def run_ours(args, rank, world, local_rank):
    import torch
    from helio_b200 import native as N
    from helio_b200 import scene as S
    from helio_b200.passes import HiZBuildPass, VirtualGeometryPass, camera_bytes, device_view

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = N.cull_lib()
    wl = build_workload(args.workload)
    sc = wl.scene
    views = wl.views
    units = sc.lod0_total * len(views)

    # Device-resident state, one pass pair per view.
    stream = torch.cuda.current_stream()
    passes = []
    for v in views:
        depth = torch.from_numpy(v.depth).to(dev)
        cam = torch.from_numpy(camera_bytes(v.camera)).to(dev)
        hz = HiZBuildPass(v.width, v.height)
        hz.prepare(depth)
        vg = VirtualGeometryPass(v.width, v.height)
        vg.prepare(S.frame_data(sc))
        passes.append((v, depth, cam, hz, vg))
    torch.cuda.synchronize()

    def step():
        for v, depth, cam, hz, vg in passes:
            hz.execute()
            vg.execute(cam, hz.publish())

    flush_buf = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    flush_read = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    flush_sink = torch.empty((), dtype=torch.float32, device=dev)

    def flush():
        # Write a buffer larger than L2, then read another one, so the timed step
        # starts with no line of its inputs in L2 and no dirty line to write back.
        flush_buf.fill_(1.0)
        torch.sum(flush_read, dim=0, out=flush_sink)

    for _ in range(max(args.warmup, 3)):
        flush()
        step()
    torch.cuda.synchronize()
    for v, depth, cam, hz, vg in passes:
        vg.device_status()
    launches0 = lib.helio_kernel_launch_count()
    step()
    torch.cuda.synchronize()
    launches_per_step = lib.helio_kernel_launch_count() - launches0

    # The step as one CUDA graph (every launch of the step, replayed by one call).
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        step()  # first launches outside capture
        torch.cuda.synchronize()
        with torch.cuda.graph(graph, stream=side):
            step()
    torch.cuda.synchronize()

    def queued():
        # A short on-device delay ahead of each timed step: the host queues the
        # whole step meanwhile, so the events time the GPU, not the enqueue.
        torch.cuda._sleep(200_000)

    for _ in range(max(args.warmup, 3)):
        flush()
        graph.replay()
    torch.cuda.synchronize()

    # Timed region: K graph replays, each bracketed by events, L2 flushed in between.
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = Clocks(local_rank)
    if world > 1:
        torch.distributed.barrier()
    clocks.start()
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush()
        queued()
        ev[k][0].record()
        graph.replay()
        ev[k][1].record()
    torch.cuda.synchronize()
    launches = launches_per_step * args.steps
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(step_ms))
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
        torch.distributed.barrier()
    value = units * args.steps * world / (total_ms / 1e3)

    # Per-kernel device time (event profiler, same steps, separate pass).
    lib.helio_profiler_reset()
    lib.helio_profiler_enable(1)
    for _ in range(args.steps):
        flush()
        queued()
        step()
    torch.cuda.synchronize()
    lib.helio_profiler_enable(0)
    prof = N.profiler_collect()
    lib.helio_profiler_reset()

    # Algorithmic bytes per launch from the step's own outputs.
    outs = []
    for v, depth, cam, hz, vg in passes:
        o = vg.outputs()
        counters = o["counters"].cpu().numpy().view(np.uint32)
        selected = o["objects"].cpu().numpy().view(np.uint32)[:, 3]
        visible = int(min(counters[0], o["capacity"]))
        outs.append((vg_algorithmic_bytes(sc, selected, visible), visible, v))
    kb = {"hiz_build": [hiz_bytes(v.width, v.height, True) for _, _, v in outs],
          "vg_select": [a["select"] for a, _, _ in outs],
          "vg_cull_test": [a["cull_test"] for a, _, _ in outs], "vg_cull_emit": [a["cull_emit"] for a, _, _ in outs]}
    kernels = {}
    tot_prof = sum(ms for _, ms in prof.values()) or 1.0
    for name, (n, ms) in prof.items():
        entry = {"launches": n, "avg_us": 1e3 * ms / max(n, 1), "share": ms / tot_prof}
        if name in kb:
            per_launch = float(np.mean(kb[name]))
            entry["algorithmic_bytes_per_launch"] = per_launch
            entry["achieved_gbs"] = per_launch / (ms / max(n, 1) / 1e3) / 1e9
        kernels[name] = entry
    dom = max((k for k in kernels if "achieved_gbs" in kernels[k]), key=lambda k: kernels[k]["share"])
    peak, peak_kind = peaks()
    traffic = None
    tfile = ROOT / "profiles" / "dram_traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get(args.workload, {}).get(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": kernels[dom]["achieved_gbs"], "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": kernels[dom]["achieved_gbs"] / peak,
                "traffic": traffic}

    # End to end through the C-ABI with host buffers.
    e2e = None
    if not args.no_e2e:
        host_depth = [torch.from_numpy(v.depth).pin_memory() for v, *_ in passes]
        host_cam = [torch.from_numpy(camera_bytes(v.camera)).pin_memory() for v, *_ in passes]
        host_cnt = [torch.empty(11, dtype=torch.int32).pin_memory() for _ in passes]
        host_out = []
        for _, _, _, _, vg in passes:
            cap = vg.outputs()["capacity"]
            host_out.append((torch.empty((max(cap, 1), 5), dtype=torch.int32).pin_memory(),
                             torch.empty((max(cap, 1), 4), dtype=torch.int32).pin_memory()))
        h2d = sum(int(t.numel()) * 4 for t in host_depth) + sum(int(t.numel()) for t in host_cam)
        d2h_total = 0

        def e2e_step():
            nonlocal d2h_total
            for i, (v, depth, cam, hz, vg) in enumerate(passes):
                depth.copy_(host_depth[i], non_blocking=True)
                cam.copy_(host_cam[i], non_blocking=True)
                hz.execute()
                vg.execute(cam, hz.publish())
                o = vg.outputs()
                host_cnt[i].copy_(o["counters"], non_blocking=True)
            torch.cuda.current_stream().synchronize()
            for i, (v, depth, cam, hz, vg) in enumerate(passes):
                o = vg.outputs()
                n = int(min(int(host_cnt[i][0]) & 0xFFFFFFFF, o["capacity"]))
                if n:
                    host_out[i][0][:n].copy_(o["indirect"][:n], non_blocking=True)
                    host_out[i][1][:n].copy_(o["draws"][:n], non_blocking=True)
                d2h_total += 44 + 36 * n
            torch.cuda.current_stream().synchronize()

        for _ in range(max(args.warmup, 3)):
            e2e_step()
        d2h_total = 0
        ee = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            flush()
            ee[k][0].record()
            e2e_step()
            ee[k][1].record()
        torch.cuda.synchronize()
        e2e_ms = float(sum(a.elapsed_time(b) for a, b in ee))
        if world > 1:
            t = torch.tensor([e2e_ms], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": units * args.steps * world / (e2e_ms / 1e3), "unit": "meshlets/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(d2h_total / args.steps),
               "ms_per_step": e2e_ms / args.steps}

    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_baseline(wl, args.cpu_seconds)

    srt = sorted(step_ms)
    line = {
        "metric": "meshlets culled/s", "value": value, "unit": "meshlets/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
        "config": {"workload": f"{args.workload}: {wl_desc(wl)}", "views": len(views),
                   "lod0_meshlets_per_view": sc.lod0_total,
                   "l2": "flushed between timed steps (256 MB write, then 256 MB read)",
                   "timing": "CUDA-graph replay of the whole step, CUDA events on the launching stream",
                   "parallelism": f"replica x{world}" if world > 1 else "single GPU"},
        "latency_ms": {"p50": srt[len(srt) // 2], "p99": srt[min(len(srt) - 1, int(math.ceil(0.99 * len(srt))) - 1)]},
        "roofline": roofline, "kernels": kernels, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": int(launches), "clocks": clk,
        "visible_draws_per_step": int(sum(vis for _, vis, _ in outs)),
    }
    return line


def wl_desc(wl) -> str:
    sc = wl.scene
    v = wl.views[0]
    return (f"{len(sc.objects)} instances x {sc.lod0_meshlets} LOD0 meshlets, {len(wl.views)} view(s), "
            f"first {v.width}x{v.height}")


def oracle_step(wl, threads: int):
    from oracle import oracle as O
    from helio_b200 import native as N

    cd = np.dtype(N.InstanceCullData)
    vis = 0
    for v in wl.views:
        levels = O.hiz_build(v.depth)
        r = O.run_view(wl.scene, v.camera, v.width, v.height, levels, v.lod_threshold_px, None, 11, threads, cd)
        vis += int(r["counters"][0])
    return vis


def cpu_baseline(wl, seconds: float) -> dict:
    """The oracle timed on this host on a bounded sample (whole steps, repeated until
    `seconds` elapse, at least one)."""
    threads = max(1, os.cpu_count() or 1)
    t0 = time.perf_counter()
    n = 0
    while True:
        oracle_step(wl, threads)
        n += 1
        if time.perf_counter() - t0 >= seconds or n >= 50:
            break
    dt = time.perf_counter() - t0
    units = wl.scene.lod0_total * len(wl.views) * n
    return {"value": units / dt, "unit": "meshlets/s", "cores": threads, "kind": "port",
            "sample": f"{n} full step(s) of the same workload (Hi-Z + select + cull, multi-threaded select/cull)",
            "seconds": dt}


def run_reference(args):
    wl = build_workload(args.workload)
    threads = max(1, os.cpu_count() or 1)
    for _ in range(args.warmup):
        oracle_step(wl, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle_step(wl, threads)
        times.append(time.perf_counter() - t0)
    units = wl.scene.lod0_total * len(wl.views)
    value = units * len(times) / sum(times)
    return {
        "metric": "meshlets culled/s", "value": value, "unit": "meshlets/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator)", "impl": "reference",
        "config": {"workload": f"{args.workload}: {wl_desc(wl)}", "views": len(wl.views),
                   "lod0_meshlets_per_view": wl.scene.lod0_total},
        "cpu_baseline": {"value": value, "unit": "meshlets/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full steps on the host cores (CPU restatement of the reference "
                                   f"shaders; the WGSL itself cannot run on this machine)"},
        "e2e": {"value": value, "unit": "meshlets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local_rank))
    line = run_ours(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
