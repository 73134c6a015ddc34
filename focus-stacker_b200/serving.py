"""Serving form: a request loop that admits focus stacks of different sizes and
frame counts against one HBM budget, streams each admitted stack's frames into
its device-resident running state as they arrive, and fuses it when its last
frame is in.

Admission is the per-request form of the reference's memory budget
(--memory-fraction, src/memory_budget.zig:3-53): a request is admitted when
the device bytes its stack will hold (fs_stack_footprint, computed without
allocating) fit in the budget left by the stacks in flight.  The stack's
pass-2 mode is the first of `modes` (by default the fused split pyramid,
then keeping the pass-1 planes, the reference's cached path, then keeping
the frames) that fits both that remainder and a cap on one stack's share of
the budget; requests wait in arrival order otherwise.  Each worker owns a context (its own streams),
so stacks in flight overlap on the device; memory comes from the device's shared stream-ordered
pool, and a worker's context budget is set to the reservation of the stack it
runs.

The report gives throughput (frame-pixels of all stacks over the makespan) and
end-to-end latency per request: arrival of the request to its fused result.
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import api


@dataclass
class StackRequest:
    rid: int
    arrival_s: float               # seconds after the start of the run
    width: int
    height: int
    frames: int
    frame_interval_s: float = 0.0  # frame i becomes available at arrival + i * interval
    level_storage: int = api.STORAGE_F32


@dataclass
class RequestResult:
    rid: int
    arrival_s: float
    admitted_s: float
    done_s: float
    frame_px: int
    pass2: str
    reserved_bytes: int
    output: Optional[np.ndarray] = None
    begin_s: float = 0.0   # stack set-up (allocation) time
    frames_s: float = 0.0  # time spent in add_frame calls (pass 1 runs asynchronously)
    finish_s: float = 0.0  # pass 2 + collapse, synchronous

    @property
    def latency_s(self) -> float:
        return self.done_s - self.arrival_s


@dataclass
class ServeReport:
    results: List[RequestResult]
    makespan_s: float
    budget_bytes: int
    peak_reserved_bytes: int
    workers: int

    def summary(self) -> dict:
        lat = np.array([r.latency_s for r in self.results])
        wait = np.array([r.admitted_s - r.arrival_s for r in self.results])
        px = sum(r.frame_px for r in self.results)
        mean_ms = lambda xs: round(float(np.mean(xs)) * 1e3, 3)  # noqa: E731
        return {
            "requests": len(self.results),
            "throughput_mpix_frames_s": round(px / self.makespan_s / 1e6, 2) if self.makespan_s > 0 else None,
            "p50_latency_ms": round(float(np.percentile(lat, 50)) * 1e3, 2),
            "p99_latency_ms": round(float(np.percentile(lat, 99)) * 1e3, 2),
            "max_latency_ms": round(float(lat.max()) * 1e3, 2),
            "p50_admission_wait_ms": round(float(np.percentile(wait, 50)) * 1e3, 2),
            "makespan_s": round(self.makespan_s, 3),
            "budget_gb": round(self.budget_bytes / 1e9, 2),
            "peak_reserved_gb": round(self.peak_reserved_bytes / 1e9, 2),
            "workers": self.workers,
            "pass2_modes": dict(collections.Counter(r.pass2 for r in self.results)),
            "mean_begin_ms": mean_ms([r.begin_s for r in self.results]),
            "mean_frames_ms": mean_ms([r.frames_s for r in self.results]),
            "mean_finish_ms": mean_ms([r.finish_s for r in self.results]),
            "busy_fraction": round(sum(r.done_s - r.admitted_s for r in self.results) /
                                   (self.makespan_s * self.workers), 3) if self.makespan_s > 0 else None,
        }


# A frame source gives, for a request, its ROI and frame i as (device buffer,
# row stride in bytes, pose).  Device buffers stay owned by the source.
RoiFn = Callable[[StackRequest], api.Rect]
FrameFn = Callable[[StackRequest, int], Tuple[object, int, object]]


class _Worker:
    def __init__(self, ctx):
        self.ctx = ctx
        self.busy = False
        self.reserved = 0  # footprint of the stack in flight
        self.mode = None   # its pass-2 mode


class StackServer:
    """max_stack_fraction caps the budget share one stack may reserve: a
    stack whose cached-planes footprint is larger runs in a smaller pass-2
    mode (frames kept and remapped again) and leaves room for the others.
    prewarm grows the device's memory pool to the budget up front."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 120 * 10**9, workers: int = 4,
                 frames_per_batch: int = 0, context_factory=None, max_stack_fraction: float = 0.25,
                 prewarm: bool = False, modes=("fused", "cache", "resident")):
        self.device = device
        self.budget = int(hbm_budget_bytes)
        self.frames_per_batch = frames_per_batch
        self.max_stack = int(self.budget * max_stack_fraction)
        self.modes = tuple(modes)
        make = context_factory or (lambda: api.Context(device, hbm_budget_bytes=self.budget))
        self.workers = [_Worker(make()) for _ in range(workers)]
        if prewarm and self.workers:
            self.workers[0].ctx.reserve(self.budget)

    def close(self):
        for w in self.workers:
            w.ctx.close()
        self.workers = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -------------------------------------------------------------- admission
    def _try_admit(self, req: StackRequest, roi: api.Rect):
        idle = [w for w in self.workers if not w.busy]
        if not idle:
            return None
        w = idle[0]
        desc = api.stack_desc(req.width, req.height, req.frames, roi, level_storage=req.level_storage,
                              frames_per_batch=self.frames_per_batch)
        # the first mode that fits what the busy workers leave of the budget
        # (bytes with the upload staging ring; the stack is begun in exactly
        # that mode)
        busy = sum(o.reserved for o in self.workers if o.busy)
        avail = min(max(0, self.budget - busy), self.max_stack)
        mode, nbytes = None, 0
        for m in self.modes:
            try:
                b = api.stack_mode_bytes(desc, m, host_frames=True)
            except api.FocusCudaError:  # mode not available for this stack (fused needs 3 levels)
                continue
            if b <= avail:
                mode, nbytes = m, b
                break
        if mode is None:
            return None
        # the stacks' memory comes from the device's shared pool, which keeps
        # freed blocks for the next stacks (trimmed by the library only when
        # an allocation finds nothing that fits): no trim here, which would
        # hand the pool's memory back and make the next stacks map it again
        w.busy = True
        w.reserved = nbytes
        w.mode = mode
        w.ctx.set_budget(max(nbytes, 1))
        return w, nbytes

    # ------------------------------------------------------------------- run
    def serve(self, requests: Sequence[StackRequest], roi_of: RoiFn, frame_of: FrameFn, torch,
              keep_outputs: bool = False) -> ServeReport:
        """Run the request stream in real time (arrival_s counted from now)
        and return the per-request results."""
        reqs = sorted(requests, key=lambda r: r.arrival_s)
        rois = {r.rid: roi_of(r) for r in reqs}
        lock = threading.Condition()
        queue: collections.deque = collections.deque()
        results: Dict[int, RequestResult] = {}
        errors: List[BaseException] = []
        peak = [0]
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731

        def run_one(w: _Worker, req: StackRequest, reserved: int, admitted: float):
            res = None
            try:
                roi = rois[req.rid]
                tb = now()
                st = api.PyramidContrastStack(w.ctx, req.width, req.height, req.frames, roi=roi,
                                              level_storage=req.level_storage,
                                              frames_per_batch=self.frames_per_batch, pass2_mode=w.mode)
                mode = st.pass2_mode
                out = torch.empty((roi.height, roi.width, 3), dtype=torch.uint8, device=f"cuda:{self.device}")
                t_begin = now() - tb
                t_frames = 0.0
                for i in range(req.frames):
                    delay = req.arrival_s + i * req.frame_interval_s - now()
                    if delay > 0:
                        time.sleep(delay)
                    buf, stride, pose = frame_of(req, i)
                    ta = now()
                    st.add_frame_device(buf, stride, pose)
                    t_frames += now() - ta
                tf = now()
                st.finish_device(out, roi.width * 3)
                t_finish = now() - tf
                st.close()
                res = RequestResult(req.rid, req.arrival_s, admitted, now(), req.frames * roi.width * roi.height,
                                    mode, reserved, out.cpu().numpy() if keep_outputs else None, t_begin, t_frames,
                                    t_finish)
            except BaseException as e:  # reported after the run
                with lock:
                    errors.append(e)
            with lock:
                if res is not None:
                    results[req.rid] = res
                w.busy = False
                w.reserved = 0
                lock.notify_all()

        threads = []
        nxt = 0
        with lock:
            while len(results) + len(errors) < len(reqs):
                t = now()
                while nxt < len(reqs) and reqs[nxt].arrival_s <= t:
                    queue.append(reqs[nxt])
                    nxt += 1
                # first come, first served: the head waits until it fits
                while queue:
                    adm = self._try_admit(queue[0], rois[queue[0].rid])
                    if adm is None:
                        break
                    w, nbytes = adm
                    req = queue.popleft()
                    peak[0] = max(peak[0], sum(x.reserved for x in self.workers if x.busy))
                    th = threading.Thread(target=run_one, args=(w, req, nbytes, now()), daemon=True)
                    th.start()
                    threads.append(th)
                wait = 0.05
                if nxt < len(reqs):
                    wait = min(wait, max(0.0, reqs[nxt].arrival_s - now()))
                lock.wait(timeout=wait if wait > 0 else 0.0005)
        for th in threads:
            th.join()
        if errors:
            raise errors[0]
        makespan = max(r.done_s for r in results.values()) - min(r.arrival_s for r in results.values())
        return ServeReport([results[r.rid] for r in reqs], makespan, self.budget, peak[0], len(self.workers))


# ----------------------------------------------------------- request streams
SIZE_MIX = ((640, 480), (1920, 1080), (4000, 3000), (6000, 4000))
LARGE = (7952, 5304)


def poisson_stream(n: int, rate_per_s: float, seed: int, large_fraction: float = 0.05, max_frames: int = 40,
                   max_large_frames: int = 143, frame_interval_s: float = 0.0,
                   level_storage: int = api.STORAGE_F32) -> List[StackRequest]:
    """n requests with exponential inter-arrival times (rate_per_s), sizes
    uniform over SIZE_MIX, frame counts uniform in [4, max_frames]; a
    large_fraction of them are 7952x5304 stacks of up to max_large_frames."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate_per_s))
        if rng.random() < large_fraction:
            (w, h), f = LARGE, int(rng.integers(4, max_large_frames + 1))
        else:
            (w, h), f = SIZE_MIX[int(rng.integers(0, len(SIZE_MIX)))], int(rng.integers(4, max_frames + 1))
        out.append(StackRequest(i, t, w, h, f, frame_interval_s, level_storage))
    return out


class SynthFramePool:
    """Device-resident synthetic frames per resolution (frame k of a stack of
    `depth` frames), shared read-only by every request of that size: request
    frames 0..F-1 are the pool's first F frames."""

    def __init__(self, ctx: api.Context, torch, device: int, seed: int, sizes, depth: Dict[Tuple[int, int], int],
                 scene: int = api.SCENE_PRODUCTION):
        self.frames: Dict[Tuple[int, int], list] = {}
        self.poses: Dict[Tuple[int, int], list] = {}
        for (w, h) in sizes:
            n = depth[(w, h)]
            fr, po = [], []
            for k in range(n):
                buf = torch.empty((h, w, 3), dtype=torch.uint8, device=f"cuda:{device}")
                po.append(api.synth_frame_device(ctx, seed, scene, w, h, k, n, buf, w * 3))
                fr.append(buf)
            self.frames[(w, h)], self.poses[(w, h)] = fr, po
        ctx.synchronize()
        self._roi_cache: Dict[Tuple[int, int, int], api.Rect] = {}

    def roi(self, req: StackRequest) -> api.Rect:
        key = (req.width, req.height, req.frames)
        if key not in self._roi_cache:
            po = self.poses[(req.width, req.height)][:req.frames]
            n = req.frames
            self._roi_cache[key] = api.compute_common_overlap_roi([True] * n, [req.width] * n, [req.height] * n, po)
        return self._roi_cache[key]

    def frame(self, req: StackRequest, i: int):
        return self.frames[(req.width, req.height)][i], req.width * 3, self.poses[(req.width, req.height)][i]
