#!/usr/bin/env python
"""Benchmark of the remap + pyramid-contrast fusion path (libfocuscuda, sm_100a).

Workload (one step = one whole stack): 30 RGB u8 frames of 7952x5304 from the
production synthetic scene (shifts up to 60 px, roll up to 0.3 deg, blur up to
8 px), remapped through their poses into the common-overlap ROI and fused with
pyramid-contrast at full pyramid depth, FP32 levels: pass 1 over all frames,
pass 2, collapse and quantise.

  value  fused MPix*frames/s = frames x ROI pixels / device time per step, all
         ranks together, frames already resident in HBM (3.8 GB per stack,
         larger than L2, so no flush is needed);
  e2e    the same metric through the public API from pinned host frames: the
         host->device copy of every frame and the device->host copy of the
         fused output are inside the timed region.  Stacks run back to back
         on one context, two in flight: each stack's pass 2, collapse and
         D2H (finish_into_async) run while the next stack's frames upload;
         the latency of one stack alone is reported beside it.

`--impl reference` times the CPU oracle (the C++ restatement of the
reference's Zig path; the Zig reference cannot be built in this image) on
the host cores for the same metric, on a bounded sample of the workload.

Multi-GPU: one process per GPU (torchrun), each rank fuses its own stack
(independent stacks, no data-path collective; weak scaling).  The CPU
baseline and the precision / serving / batched forms run at N = 1 only, so
that a scaling run holds its GPUs for the headline legs alone.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
from __graft_entry__ import load_package  # noqa: E402

METRIC = "fused MPix*frames/s (plain FP32 pyramid-contrast, remap+fuse)"
UNIT = "MPix*frames/s"

FRAMES, WIDTH, HEIGHT = 30, 7952, 5304


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=FRAMES)
    ap.add_argument("--width", type=int, default=WIDTH)
    ap.add_argument("--height", type=int, default=HEIGHT)
    ap.add_argument("--batch", type=int, default=0, help="frames per pass over per-pixel state (0 = library default)")
    ap.add_argument("--pass2-mode", default=None, choices=["cache", "resident", "refetch", "laps", "fused"],
                    help="impose the stack's pass-2 mode (default: the library's choice for the HBM budget)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the precision / serving / batched legs")
    ap.add_argument("--precision-frames", type=int, default=143,
                    help="frames of the precision-form stack (7952x5304 each; 0: skip)")
    ap.add_argument("--serving-requests", type=int, default=500, help="requests per arrival rate (serving form)")
    ap.add_argument("--serving-rates", default="20,40,60,100", help="swept Poisson arrival rates, requests/s")
    ap.add_argument("--serving-repeats", type=int, default=2,
                    help="runs per rate (independent arrival streams), so that the spread of p99 is on record")
    ap.add_argument("--serving-budget-gb", type=float, default=120.0)
    ap.add_argument("--batched-stacks", type=int, default=64, help="stacks of the batched form (0: skip)")
    ap.add_argument("--batched-budget-gb", type=float, default=130.0)
    ap.add_argument("--profile-case", action="store_true",
                    help="small case for ncu: 8 frames of 4000x3000, no e2e / CPU legs, one timed step")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + ",".join(self.FIELDS),
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) != len(self.FIELDS):
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------- algorithmic bytes
def level_sizes(w, h):
    sizes = [(w, h)]
    while w > 1 or h > 1:
        w = (w + 1) // 2 if w > 1 else 1
        h = (h + 1) // 2 if h > 1 else 1
        sizes.append((w, h))
    return sizes


def algorithmic_bytes(roi_w, roi_h, frames, k, mode="cache", storage_bytes=4):
    """Per-kernel algorithmic HBM bytes of one stack (level-streaming model):
    every tensor is written once and read once per consumer, the u8 frames are
    read once per remap, per-pixel state (weight sum, union, accumulators) is
    read and written once per batch of k frames.  mode "cache": pass 1 keeps
    the remapped frame (RGBA, 4 B) and its weight (4 B) for pass 2; "recompute":
    pass 2 remaps again into per-batch slots; "laps": pass 1 also builds the
    Gaussian/Laplacian pyramids ("image") and pass 2 only the masks and the
    blend; "fused": the same with level 0 fused into pass 1 (remap, weights,
    level-1 REDUCE, Laplacian x weight summed over frames; pass 2 divides that
    sum by the weight sum).  Returns {kernel: bytes per step} and the
    pipeline total."""
    sz = level_sizes(roi_w, roi_h)
    A = [w * h for w, h in sz]
    L = len(sz)
    batches = -(-frames // k)
    s = storage_bytes
    b = {}
    keep = 8 if mode in ("cache", "laps") else 0
    # pass 1: frame 3 B/px (+ kept planes 8 B/px); weight sum f32 and union u8
    # read+write per batch (the first batch only writes)
    b["pass1"] = frames * (3 + keep) * A[0] + batches * 10 * A[0] - 5 * A[0]
    # pass-2 re-remap (recompute mode): frame 3 B/px read, planes 8 B/px written
    b["remap_weights"] = frames * 11 * A[0] if mode == "recompute" else 0
    # level 0: planes 8 B/px read; level-1 Gaussian/mask (4 s B) + support (1 B)
    # written at 1/4 area; weight sum 4 + union 1 read and accumulator 24
    # read+write per batch
    l1 = A[1] if L > 1 else 0
    b["level0"] = frames * (8 * A[0] + (4 * s + 1) * l1) + batches * 29 * A[0]
    # levels l >= 1: read Gaussian/mask/support, write the next level;
    # mask support 1 B and accumulator 24 B per batch
    lv = 0
    for l in range(1, L - 1):
        nxt = A[l + 1] if l + 1 < L - 1 else 0
        top = A[l + 1] * 24 * batches if l + 1 == L - 1 else 0
        lv += frames * ((4 * s + 1) * (A[l] + nxt)) + batches * 25 * A[l] + top
    b["level"] = lv
    b["mask_support"] = sum(A[l] + A[l + 1] for l in range(L - 1))
    # collapse: read child accumulator (12 B), read+write parent (24 B); the
    # last step reads the base (12 B) and writes u8 RGB (3 B)
    col = 0
    for l in range(L - 1, 0, -1):
        col += 12 * A[l] + (24 * A[l - 1] if l - 1 > 0 else 15 * A[0])
    b["collapse"] = col
    b["image"] = 0
    b["blend0"] = 0
    if mode in ("laps", "fused"):
        # levels >= 1 of each frame's image pyramid: read G_l + support,
        # write the Laplacian (3s B) and G_{l+1} + support (the top one f32)
        img = 0
        for l in range(1, L - 1):
            nxt = (3 * s + 1) * A[l + 1] if l + 2 < L else 12 * A[l + 1]
            img += (3 * s + 1) * A[l] + 3 * s * A[l] + nxt
        if mode == "laps":
            # level 0 of the image pyramid: RGBA read, the f32 Laplacian
            # (12 B) and the level-1 Gaussian + support written
            img += 4 * A[0] + 12 * A[0] + (3 * s + 1) * l1
            # blend0 with the level-0 mask REDUCE: Laplacian 12 B + weight
            # 4 B read and the level-1 mask written (storage type) per frame;
            # weight sum and union support read, accumulator written once
            b["blend0"] = frames * (16 * A[0] + (s if L > 2 else 4) * l1) + 17 * A[0]
            b["level0"] = 0
        else:
            # fused pass 1: frame 3 B/px read, weight (4 B) and level-1
            # Gaussian + support (3s + 1 B at 1/4 area) written per frame;
            # weight sum f32, union u8 and the level-0 sum A_w (3 x f32) read
            # + written per batch (the first batch only writes); A_u touches
            # the window border only
            b["pass1"] = frames * (3 * A[0] + 4 * A[0] + (3 * s + 1) * l1) + batches * 34 * A[0] - 17 * A[0]
            # finalize: A_w (12) and the weight sum (4) read, acc0 (12) written
            b["blend0"] = 28 * A[0]
            # level 0: mask REDUCE of every frame from its weight and the
            # weight sum (w 4 B per frame, N and the union once), level-1
            # mask written
            b["level0"] = frames * (4 * A[0] + (s if L > 2 else 4) * l1) + 5 * A[0]
        b["image"] = frames * img
        # levels >= 1: mask REDUCE (mask read, next mask written; the top one
        # in f32; support once) and the blend of each level over all frames
        # (Laplacian 3s B (the top Gaussian 12 B) and mask read per frame,
        # accumulator 12 B written); levels 1 .. lf-1, those of at least 1184
        # 64x32 tiles, blend and REDUCE in one pass (the mask read once)
        lf = 1
        while lf + 1 < L and -(-sz[lf][0] // 64) * -(-sz[lf][1] // 32) >= 1184:
            lf += 1
        lv = 0
        for l in range(1, L):
            ms = s if l + 1 < L else 4
            if l + 1 < L:
                lv += frames * ((ms * A[l] if l >= lf else 0) + (s if l + 2 < L else 4) * A[l + 1]) + A[l]
            lv += frames * ((3 * ms) + ms) * A[l] + 12 * A[l]
        b["level"] = lv
    return b, sum(b.values())


def profile_traffic(kernel: str):
    """DRAM traffic of `kernel` per frame-pixel from a committed ncu summary
    (profiles/<kernel>_*.md, line `traffic_bytes_per_frame_px: N`), measured on
    the small profiling case; the per-launch figure scales it by the frame-pixels
    a launch processes."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for name in sorted(os.listdir(pdir)):
        if not name.startswith(kernel + "_") or not name.endswith(".md"):
            continue
        with open(os.path.join(pdir, name)) as fh:
            for line in fh:
                if line.strip().startswith("traffic_bytes_per_frame_px:"):
                    try:
                        return float(line.split(":", 1)[1].strip().split()[0])
                    except ValueError:
                        return None
    return None


def timed_steps(torch, stream, step, steps, warmup):
    """Mean device time of `step` over `steps` runs after `warmup` runs, CUDA
    events on the library's stream."""
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def precision_form(fsb, torch, dev, seed, frames_n, W=7952, H=5304, steps=2, warmup=1):
    """Precision form: the same stack with pyramid levels stored in FP32, FP16
    and BF16 (weight sums, blends and accumulators FP32 in all three).  Reports
    throughput of each and the error of the reduced forms against the FP32
    path's collapsed base on this stack (the FP32 path itself is held to 1/257
    of the FP64 oracle by the test suite, which also measures the reduced forms
    against the FP64 oracle directly)."""
    ctx = fsb.Context(dev)
    frames, poses = [], []
    for k in range(frames_n):
        buf = torch.empty((H, W, 3), dtype=torch.uint8, device=f"cuda:{dev}")
        poses.append(fsb.synth_frame_device(ctx, seed, fsb.SCENE_PRODUCTION, W, H, k, frames_n, buf, W * 3))
        frames.append(buf)
    roi = fsb.compute_common_overlap_roi([True] * frames_n, [W] * frames_n, [H] * frames_n, poses)
    out = torch.empty((roi.height, roi.width, 3), dtype=torch.uint8, device=f"cuda:{dev}")
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=f"cuda:{dev}")
    px = frames_n * roi.width * roi.height
    res = {"workload": f"{frames_n}x{W}x{H} RGB u8 synthetic focus stack (production scene), ROI "
                       f"{roi.width}x{roi.height}, frames streamed through device-resident accumulators"}
    bases = {}
    for storage in (fsb.STORAGE_F32, fsb.STORAGE_F16, fsb.STORAGE_BF16):
        name = fsb.STORAGE_NAMES[storage]
        info = {}

        def step(base=None):
            st = fsb.PyramidContrastStack(ctx, W, H, frames_n, roi=roi, level_storage=storage)
            info["pass2"] = st.pass2_mode
            if base is not None:
                st.set_base_output(base, roi.width * 3)
            for f, p in zip(frames, poses):
                st.add_frame_device(f, W * 3, p)
            st.finish_device(out, roi.width * 3)
            st.close()

        base = torch.empty((roi.height, roi.width, 3), dtype=torch.float32, device=f"cuda:{dev}")
        step(base)
        ms = timed_steps(torch, stream, step, steps, warmup)
        bases[storage] = base
        res[name] = {"value": round(px / (ms / 1e3) / 1e6, 2), "unit": UNIT, "ms_per_step": round(ms, 3),
                     "pass2": info["pass2"]}
    ref = bases[fsb.STORAGE_F32].double()
    for storage in (fsb.STORAGE_F16, fsb.STORAGE_BF16):
        d = (bases[storage].double() - ref).abs()
        mse = float((d * d).mean())
        res[fsb.STORAGE_NAMES[storage]]["vs_f32_path"] = {
            "max_abs": float(d.max()), "max_abs_lsb16": float(d.max()) * 257.0,
            "psnr_db": float("inf") if mse == 0 else 10.0 * math.log10(255.0 ** 2 / mse)}
        res[fsb.STORAGE_NAMES[storage]]["speedup_vs_f32"] = round(
            res[fsb.STORAGE_NAMES[storage]]["value"] / res["f32"]["value"], 3)
    del bases, ref
    res["vs_fp64_oracle"] = precision_error_band(fsb, torch, ctx, dev, frames, poses, W, H, roi)
    del frames
    ctx.close()
    torch.cuda.empty_cache()
    return res


def precision_error_band(fsb, torch, ctx, dev, frames, poses, W, H, roi, rows=256):
    """Error of each level storage against the FP64 oracle on a band of the
    stack: the band (full ROI width, `rows` ROI rows in the middle) is fused
    as its own ROI by the library and by the oracle evaluated in FP64 from
    the same source rows (copied back from the device frames); max-abs of
    the collapsed base in 16-bit LSBs, PSNR and the u8 difference."""
    oracle = _oracle()
    top = roi.top + (roi.height - rows) // 2
    band = fsb.Rect(roi.left, top, roi.right, top + rows)
    F = len(frames)
    host = []
    for f, p in zip(frames, poses):
        pts = [(float(x), float(y)) for x in (band.left, (band.left + band.right) / 2, band.right)
               for y in (band.top, band.bottom)]
        ys = fsb.api.inverse_map_points(p, W, H, np.array(pts))[:, 1]
        y0 = max(0, int(math.floor(min(ys))) - 4)
        y1 = min(H, int(math.ceil(max(ys))) + 5)
        img = np.zeros((H, W, 3), np.uint8)  # rows outside [y0, y1) stay untouched pages
        img[y0:y1] = f[y0:y1].cpu().numpy()
        host.append(img)
    t0 = time.perf_counter()
    ref_out, ref_base = oracle.stack_fuse(host, [p.as_dict() for p in poses], band.as_tuple(),
                                          jobs=os.cpu_count() or 1, precision=64, want_base=True, native=True)
    t_oracle = time.perf_counter() - t0
    out = {"band": f"{band.width}x{band.height} ROI rows {band.top}..{band.bottom} of the {F}-frame stack, "
                   f"{len(level_sizes(band.width, band.height))} levels; FP64 oracle {t_oracle:.1f} s on "
                   f"{os.cpu_count()} threads"}
    for storage in (fsb.STORAGE_F32, fsb.STORAGE_F16, fsb.STORAGE_BF16):
        st = fsb.PyramidContrastStack(ctx, W, H, F, roi=band, level_storage=storage)
        mode = st.pass2_mode
        base = torch.zeros((band.height, band.width, 3), dtype=torch.float32, device=f"cuda:{dev}")
        st.set_base_output(base, band.width * 3)
        for f, p in zip(frames, poses):
            st.add_frame_device(f, W * 3, p)
        fused = st.finish()
        st.close()
        err = fsb.error_vs_reference(base.cpu().numpy(), ref_base, fused, ref_out)
        out[fsb.STORAGE_NAMES[storage]] = dict({k: (round(v, 6) if isinstance(v, float) else v)
                                                for k, v in err.items()}, pass2=mode)
    del host
    return out


def serving_form(fsb, torch, dev, seed, n_requests, rates, budget_gb, workers=16, repeats=1):
    """Serving form: Poisson request streams (sizes 640x480 .. 6000x4000 with
    4-40 frames, 5 % 7952x5304 stacks of up to 143 frames) admitted against an
    HBM budget; frames are device-resident (a synthetic pool per size, as a
    GPU decoder would leave them) and streamed one at a time into each stack."""
    sv = fsb.serving
    ctx = fsb.Context(dev)
    sizes = list(sv.SIZE_MIX) + [sv.LARGE]
    depth = {s: 40 for s in sv.SIZE_MIX}
    depth[sv.LARGE] = 143
    pool = sv.SynthFramePool(ctx, torch, dev, seed, sizes, depth)
    out = {"workload": f"{n_requests} Poisson requests per rate; sizes {list(sv.SIZE_MIX)} with 4-40 frames, 5% "
                       f"7952x5304 with 4-143 frames; {budget_gb:g} GB HBM budget; {workers} workers; "
                       f"device-resident frames",
           "rates": {}}
    with sv.StackServer(dev, hbm_budget_bytes=int(budget_gb * 1e9), workers=workers, prewarm=True) as srv:
        # warm-up: one request of each size
        warm = [sv.StackRequest(i, 0.0, w, h, 4) for i, (w, h) in enumerate(sizes)]
        srv.serve(warm, pool.roi, pool.frame, torch)
        for rate in rates:
            runs = []
            for r in range(repeats):
                reqs = sv.poisson_stream(n_requests, rate, seed=seed * 1000 + int(rate) + 7919 * r)
                runs.append(srv.serve(reqs, pool.roi, pool.frame, torch).summary())
            res = dict(runs[0])
            if repeats > 1:
                res["runs"] = [{k: x[k] for k in ("p50_latency_ms", "p99_latency_ms", "throughput_mpix_frames_s",
                                                   "makespan_s")} for x in runs]
                for key in ("p50_latency_ms", "p99_latency_ms", "throughput_mpix_frames_s"):
                    res[key + "_range"] = [min(x[key] for x in runs), max(x[key] for x in runs)]
            out["rates"][f"{rate:g}"] = res
    del pool
    ctx.close()
    torch.cuda.empty_cache()
    return out


def batched_form(fsb, torch, dev, seed, n_stacks, budget_gb, reps=3):
    """Batched form: n independent stacks (4-40 frames, sizes 640x480 ..
    6000x4000, full pyramid depth each) with FP16 level storage, fused by one
    StackBatch whose schedule knobs come from the autotuner; timed over graph
    replays (frames device-resident, as a GPU decoder would leave them)."""
    sv = fsb.serving
    ctx = fsb.Context(dev, hbm_budget_bytes=int(budget_gb * 1e9))
    rng = np.random.default_rng(seed * 7 + 3)
    depth = {s: 40 for s in sv.SIZE_MIX}
    pool = sv.SynthFramePool(ctx, torch, dev, seed, sv.SIZE_MIX, depth)
    stacks, px = [], 0
    for i in range(n_stacks):
        w, h = sv.SIZE_MIX[int(rng.integers(0, len(sv.SIZE_MIX)))]
        n = int(rng.integers(4, 41))
        req = sv.StackRequest(i, 0.0, w, h, n)
        roi = pool.roi(req)
        out = torch.empty((roi.height, roi.width, 3), dtype=torch.uint8, device=f"cuda:{dev}")
        stacks.append(fsb.BatchStack(pool.frames[(w, h)][:n], pool.poses[(w, h)][:n], roi, out, w, h))
        px += n * roi.width * roi.height
    tuned = fsb.autotune.tune(ctx, stacks, reps=2, level_storage=fsb.STORAGE_F16)
    best = tuned["best"]
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=f"cuda:{dev}")
    with fsb.StackBatch(ctx, stacks, level_storage=fsb.STORAGE_F16, **best) as b:
        b.run()
        b.run()
        ms = timed_steps(torch, stream, b.run, reps, 1)
        modes = b.pass2_modes()
    res = {"workload": f"{n_stacks} stacks, frames uniform in [4, 40], sizes {list(sv.SIZE_MIX)}, "
                       f"{px / 1e6:.0f} MPix*frames per run, FP16 level storage, device-resident frames",
           "value": round(px / (ms / 1e3) / 1e6, 2), "unit": UNIT, "ms_per_run": round(ms, 3),
           "tuned": best, "graph_replay": True,
           "pass2": {m: modes.count(m) for m in set(modes)},
           "trials": [{"knobs": t["knobs"], "ms": round(t["s_per_run"] * 1e3, 3)} if "s_per_run" in t
                      else {"knobs": t["knobs"], "skipped": t["skipped"][:80]} for t in tuned["trials"]]}
    del stacks, pool
    ctx.close()
    torch.cuda.empty_cache()
    return res


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ----------------------------------------------------------- CPU baseline
# The CPU legs (cpu_baseline of this arm, and the --impl reference arm) load
# nothing of the library: poses, ROI and frames come from the oracle (its
# restatement of the reference's ROI and of the synthetic scene), and the timed
# work is the oracle's stack_fuse, built with -march=native on the host that
# runs it (strict IEEE all the same).  The sample is a full-width band of ROI
# rows of the same 30 x 7952 x 5304 stack (all frames, the same poses, the
# ROI's full width and so the same 14 pyramid levels); its source rows are the
# only ones rendered.
CPU_BAND_ROWS = 384


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def cpu_band_sample(F, W, H, seed, rows=CPU_BAND_ROWS, jobs=None):
    """Frames, poses, the stack's ROI and a band of ROI rows (left, top,
    right, bottom) for the CPU legs; frames are rendered only where the band
    samples them."""
    oracle = _oracle()
    jobs = jobs or os.cpu_count() or 1
    poses = [oracle.synth_pose(seed, oracle.SCENE_PRODUCTION, W, H, k, F) for k in range(F)]
    roi = oracle.compute_roi(poses, [W] * F, [H] * F)
    left, top, right, bottom = roi
    rows = min(rows, bottom - top)
    b_top = top + (bottom - top - rows) // 2
    band = (left, b_top, right, b_top + rows)
    frames = []
    for k, p in enumerate(poses):
        ys = [oracle.inverse_point(p, W, H, float(x), float(y))[1]
              for x in (left, (left + right) / 2, right) for y in (band[1], band[3])]
        y0 = max(0, int(math.floor(min(ys))) - 4)
        y1 = min(H, int(math.ceil(max(ys))) + 5)
        frames.append(oracle.synth_frame(seed, oracle.SCENE_PRODUCTION, W, H, k, F, rows=(y0, y1 - y0), jobs=jobs,
                                         native=True))
    return frames, poses, roi, band


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_fuse_timed(sample, steps, warmup, jobs=None):
    """Median seconds of the oracle's remap + pyramid-contrast fusion of the
    band sample (all host threads), over `steps` runs after `warmup` runs."""
    oracle = _oracle()
    frames, poses, _, band = sample
    jobs = jobs or os.cpu_count() or 1
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        oracle.stack_fuse(frames, poses, band, jobs=jobs, native=True)
        dt = time.perf_counter() - t0
        if i >= warmup:
            times.append(dt)
    return times


def band_desc(sample, F, W, H):
    band = sample[3]
    bw, bh = band[2] - band[0], band[3] - band[1]
    return (f"{F} frames of {W}x{H} (production scene, the bench's poses), ROI band {bw}x{bh} (rows "
            f"{band[1]}..{band[3]} of the stack's ROI, full ROI width, {len(level_sizes(bw, bh))} levels), oracle "
            f"stack_fuse (remap + pyramid-contrast, FP32, built -O3 -march=native -ffp-contract=off)")


def cpu_baseline(F, W, H, seed, single_thread=False):
    """cpu_baseline leg: the oracle on the band sample with every host thread
    (one warm-up, one timed run), and one thread on two of its frames."""
    oracle = _oracle()
    sample = cpu_band_sample(F, W, H, seed)
    frames, poses, _, band = sample
    cores = os.cpu_count() or 1
    times = cpu_fuse_timed(sample, steps=1, warmup=1, jobs=cores)
    t = statistics.median(times)
    px = F * (band[2] - band[0]) * (band[3] - band[1])
    out = {"value": px / t / 1e6, "unit": UNIT, "cores": cores, "kind": "port", "cpu_model": cpu_model(),
           "sample": band_desc(sample, F, W, H) + f", {cores} threads, {t:.2f} s per run"}
    if single_thread:
        t0 = time.perf_counter()
        oracle.stack_fuse(frames[:2], poses[:2], band, jobs=1, native=True)
        t1 = time.perf_counter() - t0
        out["single_thread"] = {"value": 2 * (band[2] - band[0]) * (band[3] - band[1]) / t1 / 1e6, "unit": UNIT,
                                "sample": f"the band's first 2 frames, 1 thread: {t1:.2f} s"}
    return out


def run_reference(args, rank, world):
    """--impl reference: the oracle (the C++ restatement of the reference's
    Zig path; the Zig reference cannot be built in this image) on the host
    cores, same metric and config as this arm, each step one fusion of the
    band sample.  Rank 0 alone runs it; other ranks exit without work."""
    if rank != 0:
        return
    F, W, H = args.frames, args.width, args.height
    sample = cpu_band_sample(F, W, H, args.seed)
    cores = os.cpu_count() or 1
    times = cpu_fuse_timed(sample, steps=args.steps, warmup=args.warmup, jobs=cores)
    t = statistics.mean(times)
    band = sample[3]
    px = F * (band[2] - band[0]) * (band[3] - band[1])
    value = px / t / 1e6
    cb = {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "cpu_model": cpu_model(),
          "sample": band_desc(sample, F, W, H) + f", {cores} threads, mean of {len(times)} runs after "
                    f"{args.warmup} warm-up: {t:.2f} s per run"}
    roi = sample[2]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args, roi),
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(args, roi):
    """The workload, the same in both arms: roi = (left, top, right, bottom)
    of the stack's common-overlap ROI."""
    rw, rh = roi[2] - roi[0], roi[3] - roi[1]
    return {"workload": f"{args.frames}x{args.width}x{args.height} RGB u8 synthetic focus stack "
                        "(production scene), remap + pyramid-contrast, FP32 levels",
            "frames": args.frames, "src": [args.width, args.height],
            "roi": list(roi), "levels": len(level_sizes(rw, rh)), "contrast_window": 5,
            "l2": "inputs (frames x W x H x 3 B) larger than the 126 MB L2; no flush",
            "parallelism": f"replicas x{args.gpus} (one stack per GPU)"}


# ------------------------------------------------------------------- main
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    if args.profile_case:
        args.frames, args.width, args.height, args.steps, args.warmup = 8, 4000, 3000, 1, 1
        args.no_e2e = args.no_cpu_baseline = args.no_forms = True
    fsb = load_package()
    dev = local
    F, W, H = args.frames, args.width, args.height
    ctx = fsb.Context(dev)
    frames, poses = [], []
    for k in range(F):
        buf = torch.empty((H, W, 3), dtype=torch.uint8, device=f"cuda:{dev}")
        poses.append(fsb.synth_frame_device(ctx, args.seed + rank, fsb.SCENE_PRODUCTION, W, H, k, F, buf, W * 3))
        frames.append(buf)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
    out = torch.empty((roi.height, roi.width, 3), dtype=torch.uint8, device=f"cuda:{dev}")

    mode_used = {}

    def step():
        st = fsb.PyramidContrastStack(ctx, W, H, F, roi=roi, frames_per_batch=args.batch, pass2_mode=args.pass2_mode)
        mode_used["mode"] = st.pass2_mode
        for f, p in zip(frames, poses):
            st.add_frame_device(f, W * 3, p)
        st.finish_device(out, roi.width * 3)
        st.close()

    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=f"cuda:{dev}")
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(dev)
    clocks.start()
    n0 = ctx.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    launches = (ctx.launch_count() - n0) // max(1, args.steps)
    clock_info = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    if dist:
        t = torch.tensor([ms], device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    px = F * roi.width * roi.height
    value = world * px / (ms / 1e3) / 1e6

    # per-kernel device time (CUDA events on the library's stream), one extra step
    ctx.set_kernel_timing(True)
    step()
    stats = {}
    for name in ("pass1", "image", "remap_weights", "blend0", "level0", "level", "collapse", "mask_support"):
        n, tot = ctx.kernel_stats(name)
        stats[name] = (n, tot)
    ctx.set_kernel_timing(False)
    k_default = 8 if args.batch == 0 else args.batch
    k_eff = max(1, min(k_default, 8, F))
    alg, alg_total = algorithmic_bytes(roi.width, roi.height, F, k_eff,
                                       mode_used["mode"] if mode_used["mode"] in ("cache", "laps", "fused") else "recompute")
    dom = max(stats, key=lambda n: stats[n][1])
    n_dom, ms_dom = stats[dom]
    peak, peak_kind = measured_hbm_peak()
    per_launch = alg[dom] / max(1, n_dom)
    achieved = per_launch / (ms_dom / max(1, n_dom) / 1e3) / 1e9
    traffic_fp = profile_traffic(dom)
    traffic = round(traffic_fp * px / max(1, n_dom)) if traffic_fp else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                "alg_bytes_per_launch": per_launch, "launches_per_step": n_dom,
                "avg_launch_ms": ms_dom / max(1, n_dom)}
    kernel_table = {n: {"launches": v[0], "total_ms": round(v[1], 4), "share": round(v[1] / max(1e-9, sum(
        x[1] for x in stats.values())), 4), "alg_bytes": alg[n]} for n, v in stats.items() if v[0] > 0}
    pipeline = {"alg_bytes_per_frame_pixel": alg_total / px,
                "achieved_gbs": alg_total / (ms / 1e3) / 1e9,
                "frac": (alg_total / (ms / 1e3) / 1e9) / peak}

    # end to end through the public API from pinned host memory
    e2e = None
    if not args.no_e2e:
        hframes = []
        for f in frames:
            h = torch.empty(f.shape, dtype=torch.uint8, pin_memory=True)
            h.copy_(f)
            hframes.append(h.numpy())
        houts = [torch.empty((roi.height, roi.width, 3), dtype=torch.uint8, pin_memory=True).numpy()
                 for _ in range(2)]

        def new_stack(i):
            st = fsb.PyramidContrastStack(ctx, W, H, F, roi=roi, frames_per_batch=args.batch,
                                          pass2_mode=args.pass2_mode)
            for f, p in zip(hframes, poses):
                st.add_frame_async(f, p)  # uploads queued back to back (pinned frames stay put)
            return st

        def run_stacks(n):
            # stack i's pass 2, collapse and D2H run while stack i + 1's
            # frames upload: finish_into_async, then wait on the previous one
            prev = None
            for i in range(n):
                st = new_stack(i)
                st.finish_into_async(houts[i % 2])
                if prev is not None:
                    prev.wait()
                    prev.close()
                prev = st
            prev.wait()
            prev.close()

        def single_stack():
            st = new_stack(0)
            st.finish_into(houts[0])
            st.close()

        run_stacks(3)
        # latency of one stack alone
        single_stack()
        t0 = time.perf_counter()
        for _ in range(2):
            single_stack()
        lat = (time.perf_counter() - t0) / 2
        # stacks back to back: every step still uploads its frames from pinned
        # host memory and reads its fused result back
        n_e2e = max(3, min(args.steps, 6))
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        run_stacks(n_e2e)
        dt = (time.perf_counter() - t0) / n_e2e
        if dist:
            t = torch.tensor([dt, lat], device=f"cuda:{dev}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt, lat = float(t[0].item()), float(t[1].item())
        e2e = {"value": world * px / dt / 1e6, "unit": UNIT, "h2d_bytes_per_step": F * W * H * 3,
               "d2h_bytes_per_step": roi.width * roi.height * 3, "ms_per_step": dt * 1e3,
               "stacks_in_flight": 2, "steps": n_e2e, "single_stack_latency_ms": lat * 1e3,
               "single_stack_value": world * px / lat / 1e6}
        del hframes

    forms = None
    if not args.no_forms and world == 1:
        del frames
        ctx.trim()
        torch.cuda.empty_cache()
        forms = {}
        if args.precision_frames > 0:
            forms["precision"] = precision_form(fsb, torch, dev, args.seed + rank, args.precision_frames)
        if args.serving_requests > 0:
            rates = [float(x) for x in args.serving_rates.split(",") if x]
            forms["serving"] = serving_form(fsb, torch, dev, args.seed + rank, args.serving_requests, rates,
                                            args.serving_budget_gb, repeats=args.serving_repeats)
        if args.batched_stacks > 0:
            forms["batched"] = batched_form(fsb, torch, dev, args.seed + rank, args.batched_stacks,
                                            args.batched_budget_gb)
            forms["batched"]["vs_plain_f32"] = round(forms["batched"]["value"] / value, 3)

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        cpu = cpu_baseline(F, W, H, args.seed + rank, single_thread=True)

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": workload_config(args, roi.as_tuple()), "pass2": mode_used["mode"], "frames_per_batch": k_eff,
                "e2e": e2e, "gpu_launches": launches, "clocks": clock_info, "roofline": roofline,
                "cpu_baseline": cpu, "kernels": kernel_table, "pipeline_roofline": pipeline, "forms": forms}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
