"""Autotuner of the batched form: picks, for a given set of stacks, the
schedule knobs the library exposes by timing them on the device:

  lanes             concurrent streams (graph branches) the stacks are spread
                    over; the stacks of a lane run one after another in one
                    arena, so more lanes overlap more stacks but hold more
                    device memory (one arena of the lane's largest stack each);
  frames_per_batch  frames per pass-1 launch (K, 1..8): larger K reads the
                    weight sums fewer times and gives the level launches more
                    frames (grid z) but holds K batch slots;
  pass2_mode        3: split pyramid (each frame's Laplacian pyramid kept from
                    pass 1), 4: split pyramid with level 0 blended inside
                    pass 1 (12 B per frame-pixel less to keep), 0: pass-1 planes
                    kept, 1: frames kept and remapped again, -1: the first of
                    3, 4, 0, 1 that fits the budget;
  fuse_min_tiles    level schedule: levels of at least this many 64x32 tiles
                    blend and REDUCE their masks in one pass over every frame
                    (0: the library's 1184), the smaller ones in two launches
                    with every frame in the grid;
  tail_side         level schedule: levels with both sides at most this (0:
                    64) run as the small-level tail, three launches for all of
                    them.

lanes x frames_per_batch x pass2_mode are searched first; the level schedule
(SCHEDULE_SPACE) is then searched with the best of them.

Every candidate is built as a StackBatch, run twice (direct, then captured),
and timed over `reps` graph replays; the fastest wins.  Candidates that do not
fit the context's budget are skipped.  With `cache_path`, the winner is kept
in a JSON file under the workload's signature (the stacks' sizes, frame
counts, storage and budget), and a later call with the same signature returns
it without timing.
"""
from __future__ import annotations

import itertools
import json
import os
import time
from typing import Callable, Dict, Iterable, List, Sequence

from . import api

DEFAULT_SPACE = {"lanes": (2, 4, 8), "frames_per_batch": (4, 8), "pass2_mode": (3, 4, 0)}
SCHEDULE_SPACE = {"fuse_min_tiles": (0, 296, 4294967295), "tail_side": (0, 32)}


def candidates(space: Dict[str, Iterable]) -> List[dict]:
    keys = ("lanes", "frames_per_batch", "pass2_mode")
    return [dict(zip(keys, v)) for v in itertools.product(*(tuple(space[k]) for k in keys))]


def signature(ctx: api.Context, stacks: Sequence[api.BatchStack], level_storage: int = 0) -> str:
    """Key of a workload: sorted (width, height, frames) of its stacks, the
    level storage and the context's budget in GB."""
    shapes = sorted((st.width, st.height, len(st.frames)) for st in stacks)
    return json.dumps({"stacks": shapes, "storage": level_storage, "budget_gb": round(ctx.budget() / 1e9, 1)},
                      separators=(",", ":"))


def time_batch(ctx: api.Context, stacks: Sequence[api.BatchStack], reps: int = 3, level_storage: int = 0,
               **knobs) -> dict:
    """Build, warm (direct run + capture) and time one configuration."""
    t0 = time.perf_counter()
    with api.StackBatch(ctx, stacks, level_storage=level_storage, **knobs) as b:
        b.run()
        b.run()
        setup = time.perf_counter() - t0
        t1 = time.perf_counter()
        for _ in range(reps):
            b.run()
        dt = (time.perf_counter() - t1) / reps
        modes = b.pass2_modes()
        graph = b.uses_graph
    return {"knobs": dict(knobs), "s_per_run": dt, "setup_s": setup, "graph": graph,
            "pass2": {m: modes.count(m) for m in set(modes)}}


def _load(path: str) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def tune(ctx: api.Context, stacks: Sequence[api.BatchStack], space: Dict[str, Iterable] = None, reps: int = 3,
         level_storage: int = 0, log: Callable[[str], None] = None, cache_path: str = None,
         schedule_space: Dict[str, Iterable] = None) -> dict:
    """Time every candidate of `space`, then every level schedule of
    `schedule_space` with the best of them, and return {"best": knobs,
    "trials": [...]} (from `cache_path` without timing when it holds this
    workload)."""
    key = signature(ctx, stacks, level_storage)
    if cache_path:
        hit = _load(cache_path).get(key)
        if hit is not None:
            return dict(hit, cached=True)
    trials = []
    for knobs in candidates(space or DEFAULT_SPACE):
        try:
            r = time_batch(ctx, stacks, reps=reps, level_storage=level_storage, **knobs)
        except api.FocusCudaError as e:  # does not fit the budget
            r = {"knobs": knobs, "skipped": str(e)}
        trials.append(r)
        if log:
            log(str(r))
    ok = [t for t in trials if "s_per_run" in t]
    if not ok:
        raise api.FocusCudaError(3, "no candidate fits the budget")
    best = min(ok, key=lambda t: t["s_per_run"])
    sched = schedule_space if schedule_space is not None else SCHEDULE_SPACE
    keys = ("fuse_min_tiles", "tail_side")
    for values in itertools.product(*(tuple(sched.get(k, (0,))) for k in keys)):
        if all(v == 0 for v in values):
            continue  # the library's schedule: timed above
        knobs = dict(best["knobs"], **dict(zip(keys, values)))
        try:
            r = time_batch(ctx, stacks, reps=reps, level_storage=level_storage, **knobs)
        except api.FocusCudaError as e:
            r = {"knobs": knobs, "skipped": str(e)}
        trials.append(r)
        if log:
            log(str(r))
        if "s_per_run" in r and r["s_per_run"] < best["s_per_run"]:
            best = r
    res = {"best": best["knobs"], "s_per_run": best["s_per_run"], "trials": trials}
    if cache_path:
        table = _load(cache_path)
        table[key] = {"best": res["best"], "s_per_run": res["s_per_run"]}
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1)
        os.replace(tmp, cache_path)
    return dict(res, cached=False)
