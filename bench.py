#!/usr/bin/env python
"""Benchmark of the GPU visibility path (meshlets culled per second).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step is one pass of the hot path over one synthetic frame: Hi-Z pyramid build
from each view's depth, object LOD select, meshlet frustum / cone / Hi-Z cull and
deterministic draw compaction, for every view of the workload. The metric counts
(view, LOD0 scene meshlet) pairs per second.

Workloads
  batched3 (default)  one scene of 200,000 instances x 50 LOD0 meshlets (10M), 85 views
                      (1 main 3840x2160, 4 orthographic cascades 2048^2, 16 spot 512^2,
                      64 probes 128^2), culled in ONE persistent cooperative launch; the
                      85 plain per-view pipelines are timed beside it (same inputs).
  plain2              100,000 instances x 100 LOD0 meshlets (10M), one 3840x2160 view.
  plain1 / plain0     1M meshlets at 1920x1080 / 262,144 meshlets at 1024x1024.
  serve4              the serving loop: 8 device-resident scenes (10k..2M instances x 100
                      LOD0 meshlets), a seeded Poisson stream of requests at 2,000/s, each
                      naming a scene and 1..85 views of the 85-view mix, admitted against a
                      40 GB HBM budget and batched continuously (helio_serve); reports
                      p50/p99 latency beside meshlets/s, and the same stream served one
                      request at a time through the plain single-view passes.
  instances           the instance-level passes (IndirectDispatchPass + OcclusionCullPass,
                      fused launch) over 2M draws against the 3840x2160 view; draws/s.
  shadow              the per-face shadow cull: 100,000 movable draws against 44 dirty
                      shadow faces (4 cascades, 16 spot lights, 4 point lights x 6 faces);
                      draw-face tests per second.
  vgbuild             the VG input producer: rebuild_vg_buffers on the device for the
                      largest serving scene (1.77M instance slots + 5% free slots over a
                      library of 256 meshes); slots rebuilt per second.

`value` is measured with inputs resident in HBM, the step replayed as a CUDA graph,
CUDA events on the launching stream, L2 flushed between timed steps. `e2e` runs the
same step through the C-ABI with host buffers: every view's depth and camera copied
in from pinned memory and the counters and visible draws copied out, inside the
timed region. Multi-GPU (torchrun), with no collective on the data path and time =
max over ranks: batched3 splits its 85 views across the GPUs by estimated cost, every
GPU holding the scene (strong scaling); serve4 assigns the requests of one stream to
the GPUs by cost as they arrive (weak scaling: the stream's rate grows with the GPU
count); the single-view workloads run one replica per GPU (weak scaling). `--impl reference` times the CPU restatement of the reference shaders (the
oracle) on the host cores, on rank 0 only.
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
SLEEP_CYCLES = 400_000      # on-device delay queued ahead of each timed step


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="batched3", choices=["batched3", "plain2", "plain1", "plain0", "instances", "serve4", "vgbuild", "shadow"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle check of the outputs after timing")
    ap.add_argument("--no-plain", action="store_true", help="batched3: skip the per-view plain comparison")
    ap.add_argument("--no-fold", action="store_true", help="shadow: skip the pass folded into the 85-view batch")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="bound of the CPU baseline sample")
    ap.add_argument("--requests", type=int, default=1000, help="serve4: timed requests (after --warmup x 20)")
    ap.add_argument("--rate", type=float, default=2000.0, help="serve4: arrival rate (requests/s)")
    ap.add_argument("--slots", type=int, default=2, help="serve4: batches in flight")
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
        rows = [[x.strip() for x in line.split(",")] for line in Path(self.path).read_text().splitlines()]
        rows = [r for r in rows if len(r) >= 9]
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def hiz_bytes(w: int, h: int, copy: bool) -> int:
    """Depth read, level-0 copy (unless aliased), and every level above 0 written."""
    b = 4 * w * h * (2 if copy else 1)
    for l in range(1, min(int(max(w, h)).bit_length(), 12)):
        b += 4 * max(w >> l, 1) * max(h >> l, 1)
    return b


def active_spans(scene, lod_plus_one: np.ndarray) -> tuple[int, int]:
    """(active 64-meshlet spans, tested meshlets) of one view's selected LODs."""
    obj = scene.objects
    sel = lod_plus_one.astype(np.int64)
    lod = np.maximum(sel - 1, 0)
    cnt = np.where(sel > 0, obj["lod_meshlet_counts"][np.arange(len(obj)), lod], 0).astype(np.int64)
    return int(((cnt + 63) // 64).sum()), int(cnt.sum())


def union_meshlets(scene, lods: np.ndarray) -> int:
    """Meshlets of the union over views of each object's selected LOD range."""
    obj = scene.objects
    total = 0
    counts = obj["lod_meshlet_counts"].astype(np.int64)
    for l in range(8):
        used = (lods == l + 1).any(axis=0)
        total += int(counts[used, l].sum())
    return total


# ── Workloads ─────────────────────────────────────────────────────────────────

def _u32(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)


class ParityTally:
    """Counts the views whose outputs differ from the oracle's (the check is bit-exact:
    pyramid texels compared as u32 words, every integer output element for element)
    and sums the oracle's count of decisions inside the 1e-6 relative margin band."""

    def __init__(self):
        import time as _t

        self.t0 = _t.perf_counter()
        self.views = 0
        self.bad_views = 0
        self.fields = {}
        self.marginal = {"decisions": 0, "meshlets": 0, "objects": 0}
        self.tested = 0
        self.visible = 0

    def add_view(self, got: dict, levels: list, ref: dict, pairs: dict) -> None:
        self.views += 1
        bad = []
        if len(got["levels"]) != len(levels) or any(
                not np.array_equal(a.view(np.uint32), b.view(np.uint32)) for a, b in zip(got["levels"], levels)):
            bad.append("levels")
        for gk, rk in pairs.items():
            a, b = np.asarray(got[gk]), np.asarray(ref[rk])
            if rk == "counters":
                a, b = a[:11], b[:11]
            if a.shape != b.shape or not np.array_equal(a, b):
                bad.append(gk)
        for f in bad:
            self.fields[f] = self.fields.get(f, 0) + 1
        self.bad_views += 1 if bad else 0
        st = ref["stats"]
        self.marginal["decisions"] += int(st.marginal_decisions)
        self.marginal["meshlets"] += int(st.marginal_meshlets)
        self.marginal["objects"] += int(st.marginal_objects)
        self.tested += int(st.meshlets_tested)
        self.visible += int(ref["counters"][0])

    def summary(self) -> dict:
        import time as _t

        return {"views": self.views, "mismatches": self.bad_views, "mismatched_fields": self.fields,
                "marginal_decisions": self.marginal["decisions"], "marginal_meshlets": self.marginal["meshlets"],
                "marginal_objects": self.marginal["objects"], "meshlet_tests": self.tested,
                "visible_meshlets": self.visible, "band": "1e-6 relative",
                "checker": "the oracle (CPU restatement of the reference shaders), bit-exact",
                "seconds": round(_t.perf_counter() - self.t0, 2)}


class PlainWorkload:
    """Single view through HiZBuildPass + VirtualGeometryPass (the drop-in passes)."""

    sharded = False  # one view: several GPUs run replicas

    def __init__(self, name, dev):
        import torch
        from helio_b200 import scene as S
        from helio_b200.passes import HiZBuildPass, VirtualGeometryPass, camera_bytes

        self.name = name
        self.wl = S.config({"plain2": 2, "plain1": 1, "plain0": 0}[name])
        self.scene = self.wl.scene
        self.views = self.wl.views
        self.units = self.scene.lod0_total * len(self.views)
        self.passes = []
        for v in self.views:
            depth = torch.from_numpy(v.depth).to(dev)
            cam = torch.from_numpy(camera_bytes(v.camera)).to(dev)
            hz = HiZBuildPass(v.width, v.height)
            hz.prepare(depth)
            vg = VirtualGeometryPass(v.width, v.height)
            vg.prepare(S.frame_data(self.scene))
            self.passes.append((v, depth, cam, hz, vg))

    def step(self):
        for v, depth, cam, hz, vg in self.passes:
            hz.execute()
            vg.execute(cam, hz.publish())

    def describe(self):
        v = self.views[0]
        return (f"{self.name}: {len(self.scene.objects)} instances x {self.scene.lod0_meshlets} LOD0 meshlets, "
                f"1 view {v.width}x{v.height}")

    def kernel_bytes(self) -> tuple[dict, int]:
        """Bytes an ideal implementation must move per launch, from the step's outputs:
        hiz_build = depth read + level-0 copy + levels 1.. written; vg_select = 164 B per
        object (64 B head / bounds / LOD errors, 64 B model, 16 B InstanceCullData, 4 B
        selected-LOD write, 16 B selected-range record); vg_cull_test = 24 B per work item
        (item, selected range, visibility words) + 80 B per active item (model + cull
        data) + 44 B per tested meshlet (centre, radius, cone apex, cutoff, axis);
        vg_cull_emit = 48 B per visible draw (12 B read, 36 B written)."""
        v, depth, cam, hz, vg = self.passes[0]
        o = vg.outputs()
        counters = o["counters"].cpu().numpy().view(np.uint32)
        selected = o["objects"].cpu().numpy().view(np.uint32)[: len(self.scene.objects), 3]
        visible = int(min(counters[0], o["capacity"]))
        obj, items = self.scene.objects, self.scene.work_items
        sp1 = selected.astype(np.int64)
        cnt = np.where(sp1 > 0, obj["lod_meshlet_counts"][np.arange(len(obj)), np.maximum(sp1 - 1, 0)], 0)
        n = np.clip(cnt[items["object_index"].astype(np.int64)] - items["local_meshlet_base"].astype(np.int64), 0, 64)
        tested, active = int(n.sum()), int((n > 0).sum())
        hz = hiz_bytes(v.width, v.height, True)  # the TMA form or the 128-bit-load form, whichever ran
        return {"hiz_build_tma": hz, "hiz_build": hz, "vg_select": 164 * len(obj),
                "vg_cull_test": 24 * len(items) + 80 * active + 44 * tested, "vg_cull_emit": 48 * visible}, visible

    def e2e(self):
        import torch

        host_depth = [torch.from_numpy(v.depth).pin_memory() for v, *_ in self.passes]
        host_cam = [torch.from_numpy(np.frombuffer(bytes(v.camera), np.uint8).copy()).pin_memory()
                    for v, *_ in self.passes]
        host_cnt = [torch.empty(11, dtype=torch.int32).pin_memory() for _ in self.passes]
        outs = []
        for *_, vg in self.passes:
            cap = max(vg.outputs()["capacity"], 1)
            outs.append((torch.empty((cap, 5), dtype=torch.int32).pin_memory(),
                         torch.empty((cap, 4), dtype=torch.int32).pin_memory()))
        h2d = sum(int(t.numel()) * 4 for t in host_depth) + sum(int(t.numel()) for t in host_cam)
        stats = {"d2h": 0}

        def run():
            for i, (v, depth, cam, hz, vg) in enumerate(self.passes):
                depth.copy_(host_depth[i], non_blocking=True)
                cam.copy_(host_cam[i], non_blocking=True)
                hz.execute()
                vg.execute(cam, hz.publish())
                host_cnt[i].copy_(vg.outputs()["counters"], non_blocking=True)
            torch.cuda.current_stream().synchronize()
            for i, (*_, vg) in enumerate(self.passes):
                o = vg.outputs()
                n = int(min(int(host_cnt[i][0]) & 0xFFFFFFFF, o["capacity"]))
                if n:
                    outs[i][0][:n].copy_(o["indirect"][:n], non_blocking=True)
                    outs[i][1][:n].copy_(o["draws"][:n], non_blocking=True)
                stats["d2h"] += 44 + 36 * n
            torch.cuda.current_stream().synchronize()

        return run, h2d, stats

    def parity(self, threads: int) -> dict:
        """Checker leg (after the timed region): every view's pyramid, selected LODs,
        counters, indirect args, draw records and visibility words against the oracle."""
        from oracle import oracle as O
        from helio_b200 import native as N

        res = ParityTally()
        for v, depth, cam, hz, vg in self.passes:
            levels = O.hiz_build(v.depth)
            o = vg.outputs()
            c = _u32(o["counters"])
            n = int(min(c[0], o["capacity"]))
            got = {"levels": [hz.level(l).cpu().numpy() for l in range(len(levels))], "counters": c,
                   "selected": _u32(o["objects"])[: len(self.scene.objects), 3].copy(),
                   "indirect": _u32(o["indirect"])[:n], "draws": _u32(o["draws"])[:n],
                   "visibility": _u32(o["visibility"])[: len(self.scene.work_items)]}
            ref = O.run_view(self.scene, v.camera, v.width, v.height, levels, v.lod_threshold_px, o["capacity"], 11,
                             threads, np.dtype(N.InstanceCullData))
            res.add_view(got, levels, ref, {"selected": "selected", "counters": "counters", "indirect": "indirect",
                                            "draws": "draws", "visibility": "visibility"})
        return res.summary()

    def visible_draws(self) -> int:
        tot = 0
        for *_, vg in self.passes:
            o = vg.outputs()
            tot += int(min(o["counters"].cpu().numpy().view(np.uint32)[0], o["capacity"]))
        return tot


class BatchedWorkload:
    """85 views against one device-resident scene in one cooperative launch."""

    sharded = True  # several GPUs split the 85 views

    def __init__(self, dev, with_plain=True, rank=0, world=1):
        import torch
        from helio_b200 import dist as D
        from helio_b200 import scene as S
        from helio_b200.passes import BatchedCull, HiZBuildPass, VgScene, VirtualGeometryPass, camera_bytes

        self.name = "batched3"
        self.wl = S.config(3)
        self.scene = self.wl.scene
        self.all_views = self.wl.views
        # Several GPUs: every rank holds the scene and culls its cost-balanced share of
        # the 85 views in a batch of its own (no collective on the data path).
        self.mine = D.shard_views(self.all_views, self.scene.lod0_total, world, rank) if world > 1 else \
            list(range(len(self.all_views)))
        self.views = [self.all_views[i] for i in self.mine]
        self.units = self.scene.lod0_total * len(self.views)
        self.total_units = self.scene.lod0_total * len(self.all_views)
        self.vscene = VgScene()
        self.vscene.upload(S.frame_data(self.scene))
        # Every view's depth in one device buffer (each slice starts 16-byte aligned), so
        # that the end-to-end step uploads all of them with one copy.
        sizes = [v.depth.size for v in self.views]
        self.depth_all = torch.empty(sum(sizes), dtype=torch.float32, device=dev)
        self.depths, off = [], 0
        for v, n in zip(self.views, sizes):
            d = self.depth_all[off:off + n].view(v.depth.shape)
            d.copy_(torch.from_numpy(v.depth))
            self.depths.append(d)
            off += n
        self.batch = BatchedCull(len(self.views), span_visibility=True)
        self.batch.prepare(self.vscene, [{"camera": v.camera, "depth": d, "alias_mip0": True,
                                          "lod_threshold_px": v.lod_threshold_px}
                                         for v, d in zip(self.views, self.depths)])
        torch.cuda.synchronize()
        # Launch shape chosen by the autotuner on this device, before anything is timed.
        self.tuning = self.batch.autotune(repeats=3)
        self.plain = None
        if with_plain:
            # The same 85 views through the plain single-view passes, one after another.
            self.cams = [torch.from_numpy(camera_bytes(v.camera)).to(dev) for v in self.views]
            self.hz = []
            for v, d in zip(self.views, self.depths):
                hz = HiZBuildPass(v.width, v.height, alias_mip0=True)
                hz.prepare(d)
                self.hz.append(hz)
            self.vg = VirtualGeometryPass(self.views[0].width, self.views[0].height)
            self.vg.prepare(S.frame_data(self.scene))
            torch.cuda.synchronize()
            self.plain = self.plain_step

    def step(self):
        self.batch.execute()

    def plain_step(self):
        for v, cam, hz in zip(self.views, self.cams, self.hz):
            hz.execute()
            self.vg.on_resize(v.width, v.height)
            self.vg.execute(cam, hz.publish())

    def describe(self):
        return (f"batched3: {len(self.scene.objects)} instances x {self.scene.lod0_meshlets} LOD0 meshlets "
                f"(10M), 85 views (1x 3840x2160, 4x 2048^2 orthographic, 16x 512^2 spot, 64x 128^2 probe), "
                f"one cooperative launch per GPU, Hi-Z level 0 = the view's depth")

    def outputs(self):
        lods, draws = [], 0
        for i in range(len(self.views)):
            o = self.batch.view_outputs(i)
            c = o["counters"].cpu().numpy().view(np.uint32)
            draws += int(min(c[0], o["capacity"]))
            lods.append(o["lod"].cpu().numpy()[: len(self.scene.objects)])
        return np.stack(lods), draws

    def parity(self, threads: int) -> dict:
        """Checker leg (after the timed region): every view of the batch against the
        oracle: pyramid levels, selected LOD per object, counters, indirect args and
        draw records in canonical order, and the view's active spans with their
        visibility words."""
        from oracle import oracle as O
        from helio_b200 import native as N
        from helio_b200.passes import device_view

        res = ParityTally()
        sp = self.batch.spans()
        spans, start = _u32(sp["spans"]), _u32(sp["view_span_start"])
        vis = _u32(sp["visibility"])
        items, objs = self.scene.work_items, self.scene.objects
        for i, v in enumerate(self.views):
            o = self.batch.view_outputs(i)
            c = _u32(o["counters"])
            n = int(min(c[0], o["capacity"]))
            pyr = o["pyramid"]
            got = {"levels": [device_view(pyr.levels[l], (pyr.height[l], pyr.width[l]), "<f4",
                                          (pyr.pitch[l] * 4, 4)).cpu().numpy() for l in range(pyr.mip_count)],
                   "counters": c, "lod": o["lod"].cpu().numpy()[: len(objs)].astype(np.uint32),
                   "indirect": _u32(o["indirect"])[:n], "draws": _u32(o["draws"])[:n]}
            levels = O.hiz_build(v.depth)
            ref = O.run_view(self.scene, v.camera, v.width, v.height, levels, v.lod_threshold_px, o["capacity"], 11,
                             threads, np.dtype(N.InstanceCullData))
            # The view's active spans (base below the selected LOD's count) in item order.
            sel = ref["selected"][items["object_index"]]
            lod = np.maximum(sel.astype(np.int64) - 1, 0)
            cnt = np.where(sel > 0, objs["lod_meshlet_counts"][items["object_index"], lod], 0)
            active = items["local_meshlet_base"] < cnt
            sv = spans[start[i]:start[i + 1]]
            real = (sv[:, 1] & 0x7F) > 0
            got["span_objects"] = sv[real, 3]
            got["span_visibility"] = vis[start[i]:start[i + 1]][real]
            ref["span_objects"] = items["object_index"][active]
            ref["span_visibility"] = ref["visibility"][active]
            res.add_view(got, levels, ref, {"lod": "selected", "counters": "counters", "indirect": "indirect",
                                            "draws": "draws", "span_objects": "span_objects",
                                            "span_visibility": "span_visibility"})
        return res.summary()

    def kernel_bytes(self) -> tuple[dict, int]:
        """Algorithmic bytes of the batched kernel: per view the Hi-Z (depth read + levels
        1.. written) and the per-object LOD byte, the scene's object stage once per batch
        (176 B per object: 96 B object fields, 64 B model, 16 B InstanceCullData), 44 B
        per meshlet of the union over views of each object's selected LOD range, 32 B per
        active span (16 B written, 16 B read) plus 8 B of span visibility, and 48 B per
        visible draw (12 B read, 36 B written). Split by launch: batch_kernel (phases 0-3:
        Hi-Z, LOD bytes, objects, span records written), batch_cull_kernel (phases 4-6:
        meshlets, span records read, visibility, draws)."""
        lods, visible = self.outputs()
        spans = sum(active_spans(self.scene, lods[v])[0] for v in range(len(self.views)))
        k1 = sum(hiz_bytes(v.width, v.height, False) for v in self.views)
        k1 += lods.size  # LOD bytes
        k1 += 176 * len(self.scene.objects)
        k1 += 16 * spans  # span records written by the expansion
        k2 = 44 * union_meshlets(self.scene, lods) + 24 * spans + 48 * visible
        return {"batch_kernel": k1, "batch_cull_kernel": k2}, visible

    # The two cooperative launches of one step, reported together as the step's roofline.
    step_kernels = ("batch_kernel", "batch_cull_kernel")

    def e2e(self):
        """The step through the C-ABI with host buffers: all depths in (one pinned
        copy), cameras in (one strided copy), the launch, every view's draws packed on
        the device and read back with the counters (two small copies, then two copies
        of exactly the published draws)."""
        import torch
        from helio_b200.passes import device_view

        V = len(self.views)
        host_depth = torch.from_numpy(np.concatenate([v.depth.ravel() for v in self.views])).pin_memory()
        cams = [v.camera for v in self.views]
        cap = sum(max(self.batch.view_outputs(i)["capacity"], 1) for i in range(V))
        dev = self.depth_all.device
        pk_ind = torch.empty((cap, 5), dtype=torch.int32, device=dev)
        pk_draws = torch.empty((cap, 4), dtype=torch.int32, device=dev)
        pk_off = torch.empty(V + 1, dtype=torch.int32, device=dev)
        counters = device_view(self.batch.view_outputs(0)["counters"].data_ptr(), (V, 16))
        host_ind = torch.empty((cap, 5), dtype=torch.int32).pin_memory()
        host_draws = torch.empty((cap, 4), dtype=torch.int32).pin_memory()
        host_off = torch.empty(V + 1, dtype=torch.int32).pin_memory()
        host_cnt = torch.empty((V, 16), dtype=torch.int32).pin_memory()
        h2d = int(host_depth.numel()) * 4 + 368 * V
        stats = {"d2h": 0}

        def run():
            self.depth_all.copy_(host_depth, non_blocking=True)
            self.batch.set_cameras(cams)
            self.batch.execute()
            self.batch.pack_draws(pk_ind, pk_draws, pk_off)
            host_off.copy_(pk_off, non_blocking=True)
            host_cnt.copy_(counters, non_blocking=True)
            torch.cuda.current_stream().synchronize()
            n = int(host_off[V])
            if n:
                host_ind[:n].copy_(pk_ind[:n], non_blocking=True)
                host_draws[:n].copy_(pk_draws[:n], non_blocking=True)
            stats["d2h"] += 4 * (V + 1) + 64 * V + 36 * n
            torch.cuda.current_stream().synchronize()

        return run, h2d, stats


    def e2e_pipelined(self, steps: int, warm: int) -> tuple[float, int, int]:
        """The end-to-end step over a stream of frames, pipelined as a renderer would:
        frame k+1's depths are copied in on a second stream while frame k is culled
        and its draws are copied out (two batches, one per depth buffer). Every frame
        still copies in all its depths and cameras and copies out its counters and
        exactly its published draws. Returns (ms for `steps` frames, H2D bytes per
        frame, D2H bytes per frame)."""
        import torch
        from helio_b200.passes import BatchedCull, device_view

        V = len(self.views)
        dev = self.depth_all.device
        from helio_b200.passes import camera_bytes

        # One pinned upload per frame: every view's depth, then every view's camera.
        cam_words = np.concatenate([camera_bytes(v.camera).view(np.float32) for v in self.views])
        host_in = torch.from_numpy(np.concatenate([np.concatenate([v.depth.ravel() for v in self.views]),
                                                   cam_words])).pin_memory()
        n_depth = int(self.depth_all.numel())
        host_depth = host_in
        ins = [torch.empty(host_in.numel(), dtype=torch.float32, device=dev) for _ in range(2)]
        bufs, batches = [ins[0][:n_depth], ins[1][:n_depth]], [self.batch]
        batches = []
        for buf in bufs:
            bc = BatchedCull(len(self.views), span_visibility=True)
            sizes, off, dd = [v.depth.size for v in self.views], 0, []
            for v, n in zip(self.views, sizes):
                dd.append(buf[off:off + n].view(v.depth.shape))
                off += n
            bc.prepare(self.vscene, [{"camera": v.camera, "depth": d, "alias_mip0": True,
                                      "lod_threshold_px": v.lod_threshold_px} for v, d in zip(self.views, dd)])
            buf.copy_(self.depth_all)
            bc.autotune(repeats=3)
            batches.append(bc)
        cam_dev = [x[n_depth:] for x in ins]
        batches[0].execute()
        torch.cuda.synchronize()
        visible = sum(int(batches[0].view_outputs(i)["counters"][0].item()) for i in range(V))
        cap = max(1024, 2 * visible)
        pk = [(torch.empty((cap, 5), dtype=torch.int32, device=dev), torch.empty((cap, 4), dtype=torch.int32, device=dev),
               torch.empty(V + 1, dtype=torch.int32, device=dev)) for _ in range(2)]
        cnt = [device_view(b.view_outputs(0)["counters"].data_ptr(), (V, 16)) for b in batches]
        host = [(torch.empty((cap, 5), dtype=torch.int32).pin_memory(), torch.empty((cap, 4), dtype=torch.int32).pin_memory(),
                 torch.empty(V + 1, dtype=torch.int32).pin_memory(), torch.empty((V, 16), dtype=torch.int32).pin_memory())
                for _ in range(2)]
        # Two non-default streams (the legacy default stream would serialise them).
        comp, copy = torch.cuda.Stream(), torch.cuda.Stream()
        h2d_done = [torch.cuda.Event(), torch.cuda.Event()]
        meta = [torch.cuda.Event(), torch.cuda.Event()]
        done = [torch.cuda.Event(), torch.cuda.Event()]
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        total = warm + steps
        d2h = 0
        torch.cuda.synchronize()
        with torch.cuda.stream(copy):
            ins[0].copy_(host_in, non_blocking=True)
            h2d_done[0].record(copy)
        for k in range(total):
            b = k & 1
            if k == warm:
                t0.record(comp)
                d2h = 0
            ind, drw, offs = pk[b]
            h_ind, h_drw, h_off, h_cnt = host[b]
            with torch.cuda.stream(comp):
                comp.wait_event(h2d_done[b])
                batches[b].set_cameras_device(cam_dev[b], stream=comp)
                batches[b].execute(stream=comp)
                batches[b].pack_draws(ind, drw, offs, stream=comp)
                h_off.copy_(offs, non_blocking=True)
                h_cnt.copy_(cnt[b], non_blocking=True)
                meta[b].record(comp)
            if k + 1 < total:  # the next frame's depths, into the other buffer, once its last use is done
                with torch.cuda.stream(copy):
                    if k >= 1:
                        copy.wait_event(done[1 - b])
                    ins[1 - b].copy_(host_in, non_blocking=True)
                    h2d_done[1 - b].record(copy)
            meta[b].synchronize()
            n = int(h_off[V])
            if n >= cap:
                raise RuntimeError("packed draw buffer too small")
            with torch.cuda.stream(comp):
                if n:
                    h_ind[:n].copy_(ind[:n], non_blocking=True)
                    h_drw[:n].copy_(drw[:n], non_blocking=True)
                done[b].record(comp)
            d2h += 4 * (V + 1) + 64 * V + 36 * n
        t1.record(comp)
        torch.cuda.synchronize()
        return t0.elapsed_time(t1), int(host_in.numel()) * 4, d2h // steps



class InstanceWorkload:
    """The instance-level passes (IndirectDispatchPass frustum + sub-pixel test, then
    OcclusionCullPass's 4-tap Hi-Z test against the previous frame's pyramid) in their
    fused launch over 2M draws, one per instance, of a scene with configuration 2's
    distributions (64 Gaussian blobs in a 2 km cube), seen by configuration 2's
    3840x2160 view."""

    sharded = False
    metric, unit = "instance draws culled/s", "draws/s"
    DRAWS = 2_000_000

    def __init__(self, dev):
        import torch
        from helio_b200 import passes as P
        from helio_b200 import scene as S

        self.name = "instances"
        sc = S.make_scene(S.SEED_BASE + 6, self.DRAWS, 1, 1, 1, 1000.0, 64, 20.0, lod_error_mode=1)
        self.view = S.config(2, scale=1.0).views[0]
        self.inst, self.aabbs, self.draws = sc.instances, sc.aabbs, sc.draw_calls
        self.views = [self.view]
        self.units = len(self.draws)
        up = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).to(dev)
        self.cam = up(P.camera_bytes(self.view.camera))
        self.t_inst, self.t_aabb, self.t_draw = up(self.inst), up(self.aabbs), up(self.draws)
        self.indirect = torch.zeros(len(self.draws) * 5, dtype=torch.int32, device=dev)
        self.stats = torch.zeros(8, dtype=torch.int32, device=dev)
        self.sb = P.scene_buffers(self.cam, self.t_inst, self.t_draw, self.t_aabb, self.indirect)
        self.sb.instance_count = len(self.inst)
        self.sb.draw_count = len(self.draws)
        self.depth = torch.from_numpy(self.view.depth).to(dev)
        self.hz = P.HiZBuildPass(self.view.width, self.view.height)
        self.hz.prepare(self.depth)
        self.hz.execute()
        self.fr = P.IndirectDispatchPass(self.stats)
        self.oc = P.OcclusionCullPass(self.view.width, self.view.height, self.stats)
        self.fr.prepare(self.view.camera, len(self.draws))
        self.oc.prepare(len(self.draws))
        torch.cuda.synchronize()

    def step(self):
        from helio_b200 import passes as P

        self.stats.zero_()
        P.fused_instance_cull(self.fr, self.oc, self.sb, self.hz.publish(), 1)

    def describe(self):
        return (f"instances: IndirectDispatchPass + OcclusionCullPass (fused launch) over {len(self.draws)} draws "
                f"of a 2 km scene in 64 blobs, 3840x2160 view, previous frame's Hi-Z resident")

    def kernel_bytes(self) -> tuple[dict, int]:
        """Per draw: the 20-byte draw call, the instance's bounds and flags (20 B), the
        32-byte AABB read and the 20-byte indirect record written; the Hi-Z taps are
        L2-resident and not counted."""
        visible = int(_u32(self.stats)[3]) - int(_u32(self.stats)[4])
        return {"instance_cull_fused": 92 * len(self.draws)}, visible

    def e2e(self):
        """Per frame through the C-ABI: the camera and the frame's depth copied in, the
        Hi-Z build, the fused cull, the indirect records and statistics copied out."""
        import torch
        from helio_b200 import passes as P

        host_depth = torch.from_numpy(self.view.depth).pin_memory()
        host_cam = torch.from_numpy(P.camera_bytes(self.view.camera)).pin_memory()
        host_ind = torch.empty_like(self.indirect, device="cpu").pin_memory()
        host_st = torch.empty(8, dtype=torch.int32).pin_memory()
        h2d = int(host_depth.numel()) * 4 + int(host_cam.numel())
        stats = {"d2h": 0}

        def run():
            self.depth.copy_(host_depth, non_blocking=True)
            self.cam.copy_(host_cam, non_blocking=True)
            self.hz.execute()
            self.step()
            host_ind.copy_(self.indirect, non_blocking=True)
            host_st.copy_(self.stats, non_blocking=True)
            torch.cuda.current_stream().synchronize()
            stats["d2h"] += int(self.indirect.numel()) * 4 + 32

        return run, h2d, stats

    def parity(self, threads: int) -> dict:
        """Checker leg: the indirect records and statistics against the oracle's two
        passes (the fused launch must equal frustum then occlusion)."""
        from oracle import oracle as O

        t0 = time.perf_counter()
        levels = O.hiz_build(self.view.depth)
        ind, st = O.indirect_dispatch(self.view.camera, self.inst, self.draws, self.aabbs)
        ost = O.occlusion_cull(self.view.camera, self.view.width, self.view.height, levels, self.inst, self.draws,
                               ind, st)
        g_ind = _u32(self.indirect).reshape(-1, 5)
        g_st = _u32(self.stats)
        bad = {}
        if not np.array_equal(g_ind, ind):
            bad["indirect"] = int((g_ind != ind).any(axis=1).sum())
        if not np.array_equal(g_st, st):
            bad["stats"] = 1
        return {"views": 1, "mismatches": 1 if bad else 0, "mismatched_fields": bad,
                "marginal_decisions": int(ost.marginal_decisions), "marginal_meshlets": 0, "marginal_objects": 0,
                "meshlet_tests": 0, "visible_meshlets": int(st[3]) - int(st[4]), "band": "1e-6 relative",
                "checker": "the oracle (CPU restatement of the reference shaders), bit-exact",
                "seconds": round(time.perf_counter() - t0, 2)}

    def cpu_baseline(self, seconds: float) -> dict:
        """The oracle's restatement of both passes, one host thread (as the shaders'
        per-draw work), on the whole draw list."""
        from oracle import oracle as O

        levels = O.hiz_build(self.view.depth)
        t0 = time.perf_counter()
        n = 0
        while True:
            ind, st = O.indirect_dispatch(self.view.camera, self.inst, self.draws, self.aabbs)
            O.occlusion_cull(self.view.camera, self.view.width, self.view.height, levels, self.inst, self.draws,
                             ind, st)
            n += 1
            if time.perf_counter() - t0 >= seconds or n >= 20:
                break
        dt = time.perf_counter() - t0
        return {"value": n * len(self.draws) / dt, "unit": "draws/s", "cores": 1, "kind": "port",
                "sample": f"{n} pass(es) of both passes over all {len(self.draws)} draws, one thread, {dt:.1f} s",
                "seconds": dt}


def build_workload(name, dev, with_plain, rank=0, world=1):
    if name == "instances":
        return InstanceWorkload(dev)
    return BatchedWorkload(dev, with_plain, rank, world) if name == "batched3" else PlainWorkload(name, dev)


# ── Timing ────────────────────────────────────────────────────────────────────

class Timer:
    def __init__(self, dev):
        import torch

        self.torch = torch
        self.flush_w = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
        self.flush_r = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
        self.sink = torch.empty((), dtype=torch.float32, device=dev)

    def flush(self):
        # Write a buffer larger than L2, then read another one: the step starts with
        # none of its inputs in L2 and no dirty line left to write back.
        self.flush_w.fill_(1.0)
        self.torch.sum(self.flush_r, dim=0, out=self.sink)

    def graph(self, fn):
        """fn captured as one CUDA graph (None if the capture is refused)."""
        torch = self.torch
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        try:
            with torch.cuda.stream(side):
                fn()
                torch.cuda.synchronize()
                with torch.cuda.graph(g, stream=side):
                    fn()
            torch.cuda.synchronize()
            return g
        except Exception:  # a launch that cannot be captured runs eagerly
            torch.cuda.synchronize()
            return None

    def run(self, fn, steps, warmup, graph=True):
        """Per-step device ms of fn (graph replay when possible)."""
        torch = self.torch
        g = self.graph(fn) if graph else None
        call = g.replay if g is not None else fn
        for _ in range(max(warmup, 3)):
            self.flush()
            call()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for k in range(steps):
            self.flush()
            torch.cuda._sleep(SLEEP_CYCLES)
            ev[k][0].record()
            call()
            ev[k][1].record()
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in ev], g is not None


def pct(xs, q):
    s = sorted(xs)
    return s[min(len(s) - 1, max(0, int(math.ceil(q * len(s))) - 1))]


def run_ours(args, rank, world, local_rank):
    import torch
    from helio_b200 import dist as D
    from helio_b200 import native as N

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = N.cull_lib()
    wl = build_workload(args.workload, dev, not args.no_plain, rank, world)
    # Units of the whole job per step: the 85 views once when they are split across
    # GPUs (strong scaling), every rank's replica otherwise (weak scaling).
    job_units = D.sum_over_ranks(wl.units, dev) if world > 1 else wl.units
    metric, unit = getattr(wl, "metric", "meshlets culled/s"), getattr(wl, "unit", "meshlets/s")
    timer = Timer(dev)

    wl.step()
    torch.cuda.synchronize()
    launches0 = lib.helio_kernel_launch_count()
    wl.step()
    torch.cuda.synchronize()
    launches_per_step = lib.helio_kernel_launch_count() - launches0

    clocks = Clocks(local_rank)
    if world > 1:
        torch.distributed.barrier()
    clocks.start()
    step_ms, graphed = timer.run(wl.step, args.steps, args.warmup)
    clk = clocks.stop()
    total_ms = D.max_over_ranks(sum(step_ms), dev)
    value = job_units * args.steps / (total_ms / 1e3)

    # Per-kernel device time (event profiler around every launch, eager, queued ahead).
    lib.helio_profiler_reset()
    lib.helio_profiler_enable(1)
    for _ in range(args.steps):
        timer.flush()
        torch.cuda._sleep(SLEEP_CYCLES)
        wl.step()
    torch.cuda.synchronize()
    lib.helio_profiler_enable(0)
    prof = N.profiler_collect()
    lib.helio_profiler_reset()
    kb, visible = wl.kernel_bytes()
    kernels = {}
    tot_prof = sum(ms for _, ms in prof.values()) or 1.0
    for name, (n, ms) in prof.items():
        entry = {"launches": n, "avg_us": 1e3 * ms / max(n, 1), "share": ms / tot_prof}
        if name in kb:
            entry["algorithmic_bytes_per_launch"] = float(kb[name])
            entry["achieved_gbs"] = kb[name] / (ms / max(n, 1) / 1e3) / 1e9
        kernels[name] = entry
    dom = max((k for k in kernels if "achieved_gbs" in kernels[k]), key=lambda k: kernels[k]["share"])
    step_kernels = [k for k in getattr(wl, "step_kernels", ()) if k in kernels and k in kb]
    if step_kernels:
        # A step of several launches: its bytes over the sum of their average durations.
        us = sum(kernels[k]["avg_us"] for k in step_kernels)
        dom = " + ".join(step_kernels)
        kernels[dom] = {"launches": min(kernels[k]["launches"] for k in step_kernels), "avg_us": us,
                        "share": sum(kernels[k]["share"] for k in step_kernels),
                        "algorithmic_bytes_per_launch": float(sum(kb[k] for k in step_kernels)),
                        "achieved_gbs": sum(kb[k] for k in step_kernels) / (us / 1e6) / 1e9}
    peak, peak_kind = peaks()
    traffic = None
    tfile = ROOT / "profiles" / "dram_traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get(args.workload, {}).get(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": kernels[dom]["achieved_gbs"], "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": kernels[dom]["achieved_gbs"] / peak,
                "traffic": traffic}

    extra = {}
    if hasattr(wl, "batch"):
        timer.flush()
        torch.cuda._sleep(SLEEP_CYCLES)
        wl.step()
        extra["phases_us"] = wl.batch.phase_times()
        extra["autotune"] = wl.tuning
    if getattr(wl, "plain", None) is not None:
        plain_ms, plain_graphed = timer.run(wl.plain, max(3, args.steps // 4), args.warmup)
        pm = D.max_over_ranks(sum(plain_ms), dev) / len(plain_ms)
        extra["plain_per_view"] = {"ms_per_step": pm, "value": job_units / (pm / 1e3), "unit": "meshlets/s",
                                   "graph": plain_graphed, "views": len(wl.views),
                                   "batched_speedup": pm / (total_ms / args.steps)}

    e2e = None
    if not args.no_e2e:
        run, h2d, stats = wl.e2e()
        for _ in range(max(args.warmup, 3)):
            run()
        stats["d2h"] = 0
        ee = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            timer.flush()
            ee[k][0].record()
            run()
            ee[k][1].record()
        torch.cuda.synchronize()
        e2e_ms = D.max_over_ranks(float(sum(a.elapsed_time(b) for a, b in ee)), dev)
        e2e = {"value": job_units * args.steps / (e2e_ms / 1e3), "unit": unit,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(stats["d2h"] / args.steps),
               "ms_per_step": e2e_ms / args.steps, "form": "one frame at a time (copy in, cull, copy out)"}
        if hasattr(wl, "e2e_pipelined"):
            pms, ph2d, pd2h = wl.e2e_pipelined(args.steps, max(args.warmup, 3))
            pms = D.max_over_ranks(pms, dev)
            sequential = e2e
            e2e = {"value": job_units * args.steps / (pms / 1e3), "unit": "meshlets/s",
                   "h2d_bytes_per_step": ph2d, "d2h_bytes_per_step": pd2h, "ms_per_step": pms / args.steps,
                   "form": "a stream of frames: frame k+1's depths copied in on a second stream while frame k is "
                           "culled and its draws copied out (inputs of 121 MB per frame exceed L2)",
                   "sequential": sequential}

    cpu = None
    if rank == 0 and world == 1:
        cpu = wl.cpu_baseline(args.cpu_seconds) if hasattr(wl, "cpu_baseline") else cpu_baseline(wl.wl, args.cpu_seconds)
    parity = None
    if not args.no_parity:
        # The checker, after everything timed: this rank's views against the oracle.
        torch.cuda.synchronize()
        parity = D.sum_parity(wl.parity(max(1, os.cpu_count() or 1)), dev)
    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if wl.sharded else "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator)",
        "config": {"workload": wl.describe(), "views": len(getattr(wl, "all_views", wl.views)),
                   "lod0_meshlets_per_view": wl.scene.lod0_total if hasattr(wl, "scene") else None,
                   "l2": "flushed between timed steps (256 MB write, then 256 MB read)",
                   "timing": ("CUDA-graph replay of the whole step" if graphed else "eager launches") +
                             ", CUDA events on the launching stream",
                   "parallelism": ("single GPU" if world == 1 else
                                   f"views split by estimated cost over {world} GPUs (scene replicated)"
                                   if wl.sharded else f"replica x{world}")},
        "latency_ms": {"p50": pct(step_ms, 0.5), "p99": pct(step_ms, 0.99)},
        "roofline": roofline, "kernels": kernels, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": int(launches_per_step * args.steps), "clocks": clk, "visible_draws_per_step": visible,
        "parity": parity,
    }
    line.update(extra)
    return line


# ── serve4: continuous batching of a request stream ───────────────────────────

SERVE_BUDGET = 40 * (1 << 30)
SERVE_SPANS_PER_VIEW = 1 << 19


def serve_stream(loop, lib, reqs, specs, ids, warm):
    """Replays a request stream in real time: submits each request when the host clock
    reaches its arrival, pumps the server, and records completions (releasing their
    outputs). Returns (completions by request index, batches and kernel launches after
    the first `warm` requests)."""
    done, i = {}, 0
    batches0 = loop.stats()["batches"]
    launches0 = lib.helio_kernel_launch_count()
    t0 = time.perf_counter()
    offset = reqs[0].arrival_s
    while len(done) < len(reqs):
        now = time.perf_counter() - t0
        while i < len(reqs) and reqs[i].arrival_s - offset <= now:
            loop.submit(ids[reqs[i].scene], specs[i], reqs[i].arrival_s - offset, tag=i)
            i += 1
            if i == warm:
                batches0 = loop.stats()["batches"]
                launches0 = lib.helio_kernel_launch_count()
        loop.pump(now)
        for c in loop.completions():
            done[c["tag"]] = c
            loop.release(c["request"])
        if now > 600:
            raise RuntimeError("serving run exceeded 600 s")
    return done, loop.stats()["batches"] - batches0, lib.helio_kernel_launch_count() - launches0


def run_serve(args, rank, world, local_rank):
    import torch
    from helio_b200 import dist as D
    from helio_b200 import native as N
    from helio_b200 import scene as S
    from helio_b200.passes import HiZBuildPass, ServeLoop, VgScene, VirtualGeometryPass, camera_bytes

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = N.cull_lib()
    scenes = S.serving_scenes()
    pool = S.multiview_set(S.SEED_BASE + 4)
    depths = [torch.from_numpy(v.depth).to(dev) for v in pool]
    vgs = []
    for sc in scenes:
        vs = VgScene()
        vs.upload(S.frame_data(sc))
        vgs.append(vs)
    loop = ServeLoop(hbm_budget_bytes=SERVE_BUDGET, slots=args.slots, max_views=N.HELIO_BATCH_MAX_VIEWS,
                     spans_per_view=SERVE_SPANS_PER_VIEW)
    ids = [loop.add_scene(vs) for vs in vgs]
    warm = max(3, args.warmup) * 20
    total = warm + args.requests
    # Several GPUs: one stream at world times the rate (weak scaling), each request
    # assigned on arrival to the GPU with the least estimated work so far.
    reqs = S.serving_requests(total * world, args.rate * world)
    if world > 1:
        costs = [sum(D.view_cost(pool[p].width, pool[p].height, scenes[r.scene].lod0_total) for p in r.views)
                 for r in reqs]
        owner = D.assign_online(costs, world)
        reqs = [r for r, o in zip(reqs, owner) if o == rank]
    specs = [[{"camera": pool[p].camera, "depth": depths[p], "alias_mip0": True,
               "lod_threshold_px": pool[p].lod_threshold_px} for p in r.views] for r in reqs]
    units = [scenes[r.scene].lod0_total * len(r.views) for r in reqs]
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = Clocks(local_rank)
    clocks.start()
    done, batches, launches = serve_stream(loop, lib, reqs, specs, ids, warm)
    clk = clocks.stop()
    offset = reqs[0].arrival_s
    timed = [done[k] for k in range(warm, len(reqs))]
    failed = sum(c["status"] != 0 for c in timed)
    lat = [1e3 * (c["done_s"] - c["arrival_s"]) for c in timed]
    span_s = max(c["done_s"] for c in timed) - min(c["arrival_s"] for c in timed)
    span_s = D.max_over_ranks(span_s * 1e3, dev) / 1e3
    served = sum(units[k] for k in range(warm, len(reqs)) if done[k]["status"] == 0)
    value = D.sum_over_ranks(float(served), dev) / span_s
    capacity_rps = (len(timed) - failed) / span_s

    # Latency below saturation: the same kind of stream at half the rate just served.
    low_rate = 0.5 * capacity_rps
    low_n = max(20, min(200, int(3.0 * low_rate)))
    lreqs = S.serving_requests(low_n + 20, low_rate, seed=S.SEED_BASE + 44)
    lspecs = [[{"camera": pool[p].camera, "depth": depths[p], "alias_mip0": True,
                "lod_threshold_px": pool[p].lod_threshold_px} for p in r.views] for r in lreqs]
    ldone, _, _ = serve_stream(loop, lib, lreqs, lspecs, ids, 20)
    llat = [1e3 * (ldone[k]["done_s"] - ldone[k]["arrival_s"]) for k in range(20, len(lreqs))]
    low_load = {"rate_per_s": low_rate, "requests": len(llat), "latency_ms": {"p50": pct(llat, 0.5),
                "p99": pct(llat, 0.99)}, "note": "half of the request rate served at saturation"}

    # The same timed stream served one request at a time through the plain single-view
    # passes: per-request device time (CUDA events), then the FIFO queue over the same
    # arrivals (start = max(arrival, previous finish)).
    hz = [HiZBuildPass(v.width, v.height, alias_mip0=True) for v in pool]
    for h, d in zip(hz, depths):
        h.prepare(d)
    cams = [torch.from_numpy(camera_bytes(v.camera)).to(dev) for v in pool]
    plain_ms = {}
    budget_s, t_plain = 60.0, time.perf_counter()
    for sid in ([] if args.no_plain else range(len(scenes))):
        vg = VirtualGeometryPass(pool[0].width, pool[0].height)
        vg.prepare(S.frame_data(scenes[sid]))
        mine = [k for k in range(warm, len(reqs)) if reqs[k].scene == sid]
        for k in mine:
            if time.perf_counter() - t_plain > budget_s:
                break
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for p in reqs[k].views:
                hz[p].execute()
                vg.on_resize(pool[p].width, pool[p].height)
                vg.execute(cams[p], hz[p].publish())
            b.record()
            b.synchronize()
            plain_ms[k] = a.elapsed_time(b)
        del vg
    measured = sorted(plain_ms)
    plain = None
    if measured:
        # Requests not timed (time bound) take the mean service time per (scene, view).
        per_view = {}
        for k in measured:
            per_view.setdefault(reqs[k].scene, []).append(plain_ms[k] / len(reqs[k].views))
        fin, plat = 0.0, []
        for k in range(warm, len(reqs)):
            svc = plain_ms.get(k)
            if svc is None:
                pv = per_view.get(reqs[k].scene) or [statistics.mean(plain_ms.values())]
                svc = statistics.mean(pv) * len(reqs[k].views)
            arr = 1e3 * (reqs[k].arrival_s - offset)
            fin = max(arr, fin) + svc
            plat.append(fin - arr)
        first = 1e3 * (reqs[warm].arrival_s - offset)
        plain = {"value": sum(units[warm:]) / ((fin - first) / 1e3), "unit": "meshlets/s",
                 "latency_ms": {"p50": pct(plat, 0.5), "p99": pct(plat, 0.99)},
                 "requests_timed_on_device": len(measured), "requests": len(reqs) - warm,
                 "method": "per-request device time of the plain passes (CUDA events), FIFO queue over the same "
                           "arrivals; requests beyond the 60 s timing bound use their scene's mean time per view"}

    cpu = None
    if rank == 0 and world == 1:
        small = min(range(len(scenes)), key=lambda k: len(scenes[k].objects))
        cpu = cpu_baseline(S.Workload(4, scenes[small], pool), min(args.cpu_seconds, 10.0))
        cpu["sample"] = f"scene {small} ({len(scenes[small].objects)} instances): " + cpu["sample"]
    st = loop.stats()
    return {
        "metric": "meshlets culled/s", "value": value, "unit": "meshlets/s", "n_gpus": world,
        "steps": len(timed), "warmup": warm, "ms_per_step": statistics.mean(lat), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
        "config": {"workload": "serve4: 8 scenes of " + "/".join(str(len(s.objects)) for s in scenes) +
                               " instances x 100 LOD0 meshlets; Poisson requests at "
                               f"{args.rate:g}/s per GPU, 1..85 views each from the 85-view mix; "
                               f"{args.slots} slots, {SERVE_BUDGET >> 30} GB HBM budget",
                   "requests": len(timed), "failed": failed, "batches": batches,
                   "ctas_per_slot": st["ctas_per_slot"], "peak_bytes_in_use": st["bytes_in_use"],
                   "timing": "host clock from each request's scheduled arrival to the pump that saw its "
                             "batch's completion event; value = served (view, LOD0 meshlet) pairs / (last "
                             "completion - first arrival)",
                   "l2": "not flushed: the request stream itself exceeds L2 (scenes of up to 2M instances)",
                   "parallelism": (f"requests assigned by estimated cost over {world} GPUs (scenes replicated)"
                                   if world > 1 else "single GPU")},
        "latency_ms": {"p50": pct(lat, 0.5), "p99": pct(lat, 0.99), "mean": statistics.mean(lat)},
        "capacity_requests_per_s": capacity_rps, "low_load": low_load,
        "plain_per_request": plain, "cpu_baseline": cpu, "e2e": None, "roofline": None,
        "gpu_launches": int(launches), "clocks": clk,
        "batch_requests_mean": statistics.mean(c["batch_requests"] for c in timed),
        "device": device_occupancy(timed),
    }


def device_occupancy(completions) -> dict:
    """How busy the device was over the timed requests' batches: the union of the batches'
    device intervals (CUDA events on each slot's stream) over the span from the first
    batch start to the last batch end, and the mean device time of a batch."""
    spans = sorted({(c["device_start_ms"], c["device_end_ms"]) for c in completions if c["status"] == 0})
    if not spans:
        return None
    busy, cur_s, cur_e = 0.0, spans[0][0], spans[0][1]
    for s0, e0 in spans[1:]:
        if s0 > cur_e:
            busy += cur_e - cur_s
            cur_s, cur_e = s0, e0
        else:
            cur_e = max(cur_e, e0)
    busy += cur_e - cur_s
    total = spans[-1][1] - spans[0][0] if len(spans) > 1 else busy
    total = max(total, max(e for _, e in spans) - spans[0][0])
    return {"batches": len(spans), "busy_fraction": busy / total if total > 0 else None,
            "batch_device_ms_mean": statistics.mean(e - s for s, e in spans), "span_ms": total}


# ── CPU baseline / reference arm (the oracle) ────────────────────────────────

def oracle_views(wl, views, threads: int) -> int:
    from oracle import oracle as O
    from helio_b200 import native as N

    cd = np.dtype(N.InstanceCullData)
    vis = 0
    for v in views:
        levels = O.hiz_build(v.depth)
        r = O.run_view(wl.scene, v.camera, v.width, v.height, levels, v.lod_threshold_px, None, 11, threads, cd)
        vis += int(r["counters"][0])
    return vis


def sample_views(wl, k: int):
    """Every 5th view (offset by k) of a many-view workload; all views otherwise."""
    return wl.views if len(wl.views) < 10 else wl.views[k % 5::5]


def cpu_baseline(wl, seconds: float) -> dict:
    threads = max(1, os.cpu_count() or 1)
    t0 = time.perf_counter()
    n_units = 0
    k = 0
    while True:
        views = sample_views(wl, k)
        oracle_views(wl, views, threads)
        n_units += wl.scene.lod0_total * len(views)
        k += 1
        if time.perf_counter() - t0 >= seconds or k >= 50:
            break
    dt = time.perf_counter() - t0
    return {"value": n_units / dt, "unit": "meshlets/s", "cores": threads, "kind": "port",
            "sample": f"{k} step(s) of {len(sample_views(wl, 0))} view(s) each (Hi-Z + select + cull per view, "
                      f"multi-threaded select / cull), {dt:.1f} s", "seconds": dt}


# ── vgbuild: the VG input producer ────────────────────────────────────────────

VGBUILD_FREE_SLOTS = 0.05


def vgbuild_library():
    from helio_b200 import scene as S

    counts = S.serving_counts()
    k = max(range(len(counts)), key=lambda i: counts[i])
    return S.library_from_scene(S.serving_scene(k), free_slots=VGBUILD_FREE_SLOTS, seed=7), counts[k]


def vgbuild_bytes(lib, out) -> int:
    """Algorithmic bytes of one rebuild: each slot's mesh index and instance read; each
    mesh record read once; descriptors read and written; objects, instances and work
    items written."""
    return int(lib.slot_mesh.nbytes + lib.slot_instances.nbytes + 128 * len(lib.meshes) +
               2 * out["meshlets"].nbytes + out["objects"].nbytes + out["instances"].nbytes +
               out["work_items"].nbytes)


def vgbuild_cpu(lib, seconds: float, steps: int | None = None) -> tuple[float, int, float]:
    """Oracle rebuilds of the library (single thread, as the reference's rebuild):
    returns (slots/s, runs, total seconds)."""
    from oracle import oracle as O

    O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances)
    t, runs = 0.0, 0
    while (steps is None and (t < seconds or runs < 1)) or (steps is not None and runs < steps):
        t0 = time.perf_counter()
        O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances)
        t += time.perf_counter() - t0
        runs += 1
    return len(lib.slot_mesh) * runs / t, runs, t


def run_build(args, rank, world, local_rank):
    import torch
    from helio_b200 import dist as D
    from helio_b200 import native as N
    from helio_b200.passes import VgBuilder

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib_n = N.cull_lib()
    lib, instances = vgbuild_library()

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).to(dev)

    d = [up(lib.pool), up(lib.meshes), up(lib.slot_mesh), up(lib.slot_instances)]
    b = VgBuilder()

    def step():
        b.run(*d)

    step()
    torch.cuda.synchronize()
    out = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in b.outputs().items()}
    launches0 = lib_n.helio_kernel_launch_count()
    step()
    launches_per_step = lib_n.helio_kernel_launch_count() - launches0
    timer = Timer(dev)
    clocks = Clocks(local_rank)
    if world > 1:
        torch.distributed.barrier()
    clocks.start()
    # The rebuild reads its totals back once (to size its outputs): eager, not a graph.
    step_ms, _ = timer.run(step, args.steps, args.warmup, graph=False)
    clk = clocks.stop()
    total_ms = D.max_over_ranks(sum(step_ms), dev)
    slots = len(lib.slot_mesh)
    value = slots * args.steps * world / (total_ms / 1e3)

    lib_n.helio_profiler_reset()
    lib_n.helio_profiler_enable(1)
    for _ in range(args.steps):
        timer.flush()
        step()
    torch.cuda.synchronize()
    lib_n.helio_profiler_enable(0)
    prof = N.profiler_collect()
    lib_n.helio_profiler_reset()
    n, ms = prof["vg_build"]
    alg = vgbuild_bytes(lib, out)
    achieved = alg / (ms / n / 1e3) / 1e9
    peak, peak_kind = peaks()
    tfile = ROOT / "profiles" / "dram_traffic.json"
    traffic = json.loads(tfile.read_text()).get("vgbuild", {}).get("vg_build") if tfile.exists() else None
    roofline = {"bound": "hbm", "kernel": "vg_build", "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "note": "the six launches of one rebuild and its two read-backs (totals, error word), between one "
                        "pair of CUDA events"}

    e2e = None
    if not args.no_e2e:
        # The per-frame part (slot arrays) copied in from pinned host memory each step;
        # the pool and mesh records stay resident; then the rebuild.
        hs = [torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).pin_memory()
              for a in (lib.slot_mesh, lib.slot_instances)]

        def run_e2e():
            d[2].copy_(hs[0], non_blocking=True)
            d[3].copy_(hs[1], non_blocking=True)
            b.run(*d)

        for _ in range(max(args.warmup, 3)):
            run_e2e()
        ee = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            timer.flush()
            ee[k][0].record()
            run_e2e()
            ee[k][1].record()
        torch.cuda.synchronize()
        e2e_ms = D.max_over_ranks(float(sum(a.elapsed_time(z) for a, z in ee)), dev)
        e2e = {"value": slots * args.steps * world / (e2e_ms / 1e3), "unit": "slots/s",
               "h2d_bytes_per_step": int(sum(h.numel() for h in hs)), "d2h_bytes_per_step": 48 + 4,
               "ms_per_step": e2e_ms / args.steps,
               "form": "slot arrays copied in from pinned host memory, then the rebuild (its totals and error "
                       "word read back)"}
    cpu = None
    if rank == 0 and world == 1:
        v, runs, t = vgbuild_cpu(lib, args.cpu_seconds)
        cpu = {"value": v, "unit": "slots/s", "cores": 1, "kind": "port",
               "sample": f"{runs} oracle rebuild(s) of the full library ({slots} slots), {t:.1f} s"}
    return {
        "metric": "VG slots rebuilt/s", "value": value, "unit": "slots/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generator)",
        "config": {"workload": f"vgbuild: the largest serving scene ({instances} instances x 100 LOD0 meshlets) as "
                               f"{slots} dense slots ({VGBUILD_FREE_SLOTS:.0%} free) over {len(lib.meshes)} meshes "
                               f"and {len(lib.pool)} pool descriptors",
                   "outputs": {"descriptors": len(out["meshlets"]) // 64, "objects": len(out["objects"]) // 128,
                               "work_items": len(out["work_items"]) // 8, "max_draw_count": out["max_draw_count"]},
                   "l2": "flushed between timed steps (256 MB write, then 256 MB read)",
                   "timing": "eager launches (the rebuild synchronises once to size its outputs), CUDA events on "
                             "the launching stream",
                   "parallelism": f"replica x{world}" if world > 1 else "single GPU"},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches_per_step * args.steps),
        "clocks": clk,
    }


# ── shadow: the per-face shadow cull ──────────────────────────────────────────

SHADOW_DRAWS = 100_000


def shadow_workload():
    """Faces and draws of the shadow workload (seeded synthetic inputs)."""
    from helio_b200 import scene as S

    mats, nf = S.shadow_faces(11)
    inst, src = S.shadow_draws(11, SHADOW_DRAWS, SHADOW_DRAWS)
    dirty = np.zeros(256, np.uint32)
    dirty[:nf] = 1
    return mats, nf, inst, src, dirty


def shadow_cpu(mats, nf, inst, src, dirty, seconds: float, steps: int | None = None):
    from oracle import oracle as O

    t, runs = 0.0, 0
    while (steps is None and (t < seconds or runs < 1)) or (steps is not None and runs < steps):
        t0 = time.perf_counter()
        O.shadow_cull(mats, inst, src, dirty, nf)
        t += time.perf_counter() - t0
        runs += 1
    return len(src) * nf * runs / t, runs, t


def run_shadow(args, rank, world, local_rank):
    import torch
    from helio_b200 import dist as D
    from helio_b200 import native as N
    from helio_b200.passes import ShadowCullPass

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib_n = N.cull_lib()
    mats, nf, inst, src, dirty = shadow_workload()

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    d = [up(mats), up(inst.view(np.uint8)), up(src.view(np.int32)), up(dirty.view(np.int32))]
    p = ShadowCullPass()
    p.prepare(*d, nf)
    p.execute()
    torch.cuda.synchronize()
    visible = int(p.outputs()["face_counts"].cpu().numpy().view(np.uint32)[:nf].sum())
    launches0 = lib_n.helio_kernel_launch_count()
    p.execute()
    launches_per_step = lib_n.helio_kernel_launch_count() - launches0
    timer = Timer(dev)
    clocks = Clocks(local_rank)
    clocks.start()
    step_ms, graphed = timer.run(p.execute, args.steps, args.warmup)
    clk = clocks.stop()
    total_ms = D.max_over_ranks(sum(step_ms), dev)
    tests = len(src) * nf
    value = tests * args.steps * world / (total_ms / 1e3)
    # Algorithmic bytes: each draw's 20-byte record and its instance's 16-byte sphere
    # read once, each visible (draw, face) record written (up to 4096 a face).
    stored = int(np.minimum(p.outputs()["face_counts"].cpu().numpy().view(np.uint32)[:nf], 4096).sum())
    alg = len(src) * 36 + stored * 20 + 256 * 4
    achieved = alg / (total_ms / args.steps / 1e3) / 1e9
    peak, peak_kind = peaks()
    roofline = {"bound": "hbm", "kernel": "shadow_cull", "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                "note": "three launches per step (graph replay); latency-bound at this size"}
    e2e = None
    if not args.no_e2e:
        hs = torch.from_numpy(np.ascontiguousarray(src.view(np.int32))).pin_memory()
        out_counts = torch.empty(256, dtype=torch.int32).pin_memory()

        def run_e2e():
            d[2].copy_(hs, non_blocking=True)
            p.execute()
            out_counts.copy_(p.outputs()["face_counts"], non_blocking=True)

        for _ in range(max(args.warmup, 3)):
            run_e2e()
        ee = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            timer.flush()
            ee[k][0].record()
            run_e2e()
            ee[k][1].record()
        torch.cuda.synchronize()
        e2e_ms = D.max_over_ranks(float(sum(a.elapsed_time(z) for a, z in ee)), dev)
        e2e = {"value": tests * args.steps * world / (e2e_ms / 1e3), "unit": "draw-face tests/s",
               "h2d_bytes_per_step": int(hs.numel() * 4), "d2h_bytes_per_step": 256 * 4,
               "ms_per_step": e2e_ms / args.steps,
               "form": "the draw records copied in from pinned host memory, the cull, the 256 counts copied out"}
    folded = None if args.no_fold else shadow_fold_times(timer, dev, p, args.steps, args.warmup)
    cpu = None
    if rank == 0 and world == 1:
        v, runs, t = shadow_cpu(mats, nf, inst, src, dirty, args.cpu_seconds)
        cpu = {"value": v, "unit": "draw-face tests/s", "cores": 1, "kind": "port",
               "sample": f"{runs} oracle run(s) of the full workload, {t:.1f} s"}
    return {
        "metric": "shadow draw-face tests/s", "value": value, "unit": "draw-face tests/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
        "config": {"workload": f"shadow: {len(src)} movable draws over {len(inst)} instances x {nf} dirty faces "
                               "(4 orthographic cascades, 16 spot, 4 point lights x 6)",
                   "visible_draw_faces": visible,
                   "l2": "flushed between timed steps (256 MB write, then 256 MB read)",
                   "timing": ("CUDA-graph replay" if graphed else "eager launches") + ", CUDA events",
                   "parallelism": f"replica x{world}" if world > 1 else "single GPU"},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches_per_step * args.steps),
        "clocks": clk, "folded": folded,
    }


def shadow_fold_times(timer, dev, p, steps: int, warmup: int) -> dict:
    """Device ms per step (median, graph replay, L2 flushed) of the 85-view batch of the
    batched3 workload alone, of the batch followed by the standalone shadow pass `p`, and
    of the batch with `p` folded into its launches (helio_batch_attach_shadow)."""
    import torch
    from helio_b200 import scene as S
    from helio_b200.passes import BatchedCull, VgScene

    wl = S.config(3)
    vs = VgScene()
    vs.upload(S.frame_data(wl.scene))
    depths = [torch.from_numpy(v.depth).to(dev) for v in wl.views]
    b = BatchedCull(len(wl.views))
    b.prepare(vs, [{"camera": v.camera, "depth": t, "alias_mip0": True, "lod_threshold_px": v.lod_threshold_px}
                   for v, t in zip(wl.views, depths)])
    out = {"form": "85-view batch of the batched3 workload (two cooperative launches) with the shadow step"}
    for name, fn in (("batch_ms", b.execute), ("batch_then_shadow_ms", lambda: (b.execute(), p.execute()))):
        ms, _ = timer.run(fn, steps, warmup)
        out[name] = float(np.median(ms))
    b.attach_shadow(p)
    ms, _ = timer.run(b.execute, steps, warmup)
    out["batch_with_folded_shadow_ms"] = float(np.median(ms))
    b.status()
    b.attach_shadow(None)
    return out


def run_reference(args):
    from helio_b200 import scene as S

    if args.workload == "shadow":
        mats, nf, inst, src, dirty = shadow_workload()
        for _ in range(args.warmup):
            shadow_cpu(mats, nf, inst, src, dirty, 0.0, steps=1)
        v, runs, t = shadow_cpu(mats, nf, inst, src, dirty, 0.0, steps=args.steps)
        return {"metric": "shadow draw-face tests/s", "value": v, "unit": "draw-face tests/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / runs,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded generator)", "impl": "reference", "config": {"workload": "shadow"},
                "cpu_baseline": {"value": v, "unit": "draw-face tests/s", "cores": 1, "kind": "port",
                                 "sample": "each step: the full workload through the oracle's restatement of "
                                           "shadow_cull.wgsl (single thread)"},
                "e2e": {"value": v, "unit": "draw-face tests/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}

    if args.workload == "vgbuild":
        lib, _ = vgbuild_library()
        for _ in range(args.warmup):
            vgbuild_cpu(lib, 0.0, steps=1)
        v, runs, t = vgbuild_cpu(lib, 0.0, steps=args.steps)
        return {"metric": "VG slots rebuilt/s", "value": v, "unit": "slots/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / runs, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generator)",
                "impl": "reference", "config": {"workload": "vgbuild", "slots": len(lib.slot_mesh)},
                "cpu_baseline": {"value": v, "unit": "slots/s", "cores": 1, "kind": "port",
                                 "sample": "each step: one rebuild of the full library by the oracle's restatement "
                                           "of rebuild_vg_buffers (single thread, as the reference)"},
                "e2e": {"value": v, "unit": "slots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "instances":
        from oracle import oracle as O

        sc = S.make_scene(S.SEED_BASE + 6, InstanceWorkload.DRAWS, 1, 1, 1, 1000.0, 64, 20.0, lod_error_mode=1)
        view = S.config(2).views[0]
        levels = O.hiz_build(view.depth)

        def one():
            ind, st = O.indirect_dispatch(view.camera, sc.instances, sc.draw_calls, sc.aabbs)
            O.occlusion_cull(view.camera, view.width, view.height, levels, sc.instances, sc.draw_calls, ind, st)

        for _ in range(args.warmup):
            one()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            one()
        t = time.perf_counter() - t0
        v = args.steps * len(sc.draw_calls) / t
        return {"metric": "instance draws culled/s", "value": v, "unit": "draws/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded generator)", "impl": "reference", "config": {"workload": "instances"},
                "cpu_baseline": {"value": v, "unit": "draws/s", "cores": 1, "kind": "port",
                                 "sample": "each step: all draws through the oracle's restatement of "
                                           "indirect_dispatch.wgsl and occlusion_cull.wgsl (single thread)"},
                "e2e": {"value": v, "unit": "draws/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "serve4":
        # The reference has no serving loop; its per-view cull, restated, on the smallest
        # serving scene and the 85-view mix.
        scenes = S.serving_scenes()
        small = min(scenes, key=lambda sc: len(sc.objects))
        wl = S.Workload(4, small, S.multiview_set(S.SEED_BASE + 4))
    else:
        wl = S.config({"batched3": 3, "plain2": 2, "plain1": 1, "plain0": 0}[args.workload])
    threads = max(1, os.cpu_count() or 1)
    for k in range(args.warmup):
        oracle_views(wl, sample_views(wl, k), threads)
    times, units = [], 0
    for k in range(args.steps):
        views = sample_views(wl, k)
        t0 = time.perf_counter()
        oracle_views(wl, views, threads)
        times.append(time.perf_counter() - t0)
        units += wl.scene.lod0_total * len(views)
    value = units / sum(times)
    sample = (f"each step: {len(sample_views(wl, 0))} of {len(wl.views)} views (every 5th, rotating) of the same "
              f"workload" if len(wl.views) >= 10 else "each step: the full workload")
    return {
        "metric": "meshlets culled/s", "value": value, "unit": "meshlets/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator)", "impl": "reference",
        "config": {"workload": args.workload, "views": len(wl.views), "lod0_meshlets_per_view": wl.scene.lod0_total},
        "cpu_baseline": {"value": value, "unit": "meshlets/s", "cores": threads, "kind": "port",
                         "sample": sample + "; CPU restatement of the reference shaders (the WGSL itself cannot "
                                            "run on this machine)"},
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
        from helio_b200 import dist as D

        D.init("nccl", timeout_s=120)
    if args.workload == "serve4":
        line = run_serve(args, rank, world, local_rank)
    elif args.workload == "vgbuild":
        line = run_build(args, rank, world, local_rank)
    elif args.workload == "shadow":
        line = run_shadow(args, rank, world, local_rank)
    else:
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
