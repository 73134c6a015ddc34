"""Autotuner of the batched form: picks, for a given set of stacks, the
schedule knobs the library exposes by timing them on the device:

  lanes             concurrent streams (graph branches) the stacks are spread over;
  frames_per_batch  frames per pass over the per-pixel state (K, 1..8): larger
                    K reads the accumulators and weight sums fewer times but
                    holds K level slots;
  pass2_mode        0: keep the pass-1 planes for pass 2 (8 B per frame-pixel
                    of memory), 1: keep only the frames and remap them again,
                    -1: per stack, the planes while the budget allows.

Every candidate is built as a StackBatch, run twice (direct, then captured),
and timed over `reps` graph replays; the fastest wins.  Candidates that do not
fit the context's budget are skipped.  Results are plain dicts, so a caller can
store them per workload signature and skip the search next time.
"""
from __future__ import annotations

import itertools
import time
from typing import Callable, Dict, Iterable, List, Sequence

from . import api

DEFAULT_SPACE = {"lanes": (4, 8, 16), "frames_per_batch": (8,), "pass2_mode": (-1, 1)}


def candidates(space: Dict[str, Iterable]) -> List[dict]:
    keys = ("lanes", "frames_per_batch", "pass2_mode")
    return [dict(zip(keys, v)) for v in itertools.product(*(tuple(space[k]) for k in keys))]


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


def tune(ctx: api.Context, stacks: Sequence[api.BatchStack], space: Dict[str, Iterable] = None, reps: int = 3,
         level_storage: int = 0, log: Callable[[str], None] = None) -> dict:
    """Time every candidate of `space` and return {"best": knobs, "trials": [...]}."""
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
    return {"best": best["knobs"], "s_per_run": best["s_per_run"], "trials": trials}
