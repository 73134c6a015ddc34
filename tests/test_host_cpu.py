"""CPU tests of the library's host logic and closed forms (no GPU needed)."""
import ctypes
import math
import os

import numpy as np
import pytest

import oracle
from __graft_entry__ import load_package

fsb = load_package()


def test_library_exports_every_declared_symbol():
    import re
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "focuscuda.h")).read()
    declared = set(re.findall(r"\b(fs_[a-z0-9_]+)\s*\(", hdr)) - {"fs_frame_fetch_cb"}
    assert declared == set(fsb._lib.EXPORTED)
    L = fsb._lib.lib()
    for name in declared:
        assert getattr(L, name) is not None


def test_status_strings_and_version():
    L = fsb._lib.lib()
    assert L.fs_api_version() == 1
    assert L.fs_status_string(0) == b"ok"
    assert L.fs_status_string(3) == b"device memory budget exceeded"


def test_stack_entry_points_reject_null_handles():
    # argument checks run before any CUDA call, so they hold without a GPU
    L = fsb._lib.lib()
    invalid = 1  # FS_ERR_INVALID
    pixels = np.zeros(16, np.uint8)
    out = np.zeros(16, np.uint8)
    assert L.fs_stack_wait(None) == invalid
    assert L.fs_stack_add_frame_async(None, pixels.ctypes.data, 16, None) == invalid
    assert L.fs_stack_add_frame(None, pixels.ctypes.data, 16, None) == invalid
    cb = ctypes.cast(None, fsb._lib.FETCH_CB)
    assert L.fs_stack_finish_async(None, cb, None, out.ctypes.data, 16) == invalid
    assert L.fs_stack_finish(None, cb, None, out.ctypes.data, 16) == invalid
    assert L.fs_ctx_set_level_schedule(None, 0, 0) == invalid
    assert L.fs_check_normalise(None, None, None, None, 0) == invalid


def test_context_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(fsb.FocusCudaError) as e:
        fsb.Context(0)
    assert e.value.code == "FS_ERR_NO_DEVICE"


def test_parse_method_and_window():
    assert fsb.parse_method("cuda-pyramid-contrast") is fsb.Method.CUDA_PYRAMID_CONTRAST
    assert fsb.parse_method("pyramid-contrast") is fsb.Method.PYRAMID_CONTRAST
    with pytest.raises(ValueError):
        fsb.parse_method("pyramid")
    assert fsb.parse_window_size("7") == 7
    for bad in ("4", "1", "0", "x"):
        with pytest.raises(ValueError):
            fsb.parse_window_size(bad)


def _random_poses(rng, n, w, kinds=("basic",)):
    poses = []
    f = (w / 2) / math.tan(math.radians(25))
    for i in range(n):
        kind = kinds[i % len(kinds)]
        p = fsb.ImagePose(yaw=math.atan(rng.uniform(-60, 60) / f), pitch=math.atan(rng.uniform(-60, 60) / f),
                          roll=math.radians(rng.uniform(-0.3, 0.3)), hfov_delta=rng.uniform(-0.2, 0.2))
        if kind == "lens":
            p.radial_a, p.radial_b, p.radial_c = rng.uniform(-0.02, 0.02, 3)
            p.center_shift_x, p.center_shift_y = rng.uniform(-3, 3, 2)
        if kind == "shift":
            p.center_shift_x, p.center_shift_y = rng.uniform(-3, 3, 2)
        if kind == "trans":
            p.trans_x, p.trans_y, p.trans_z = rng.uniform(-3, 3), rng.uniform(-3, 3), rng.uniform(-0.02, 0.02)
            p.translation_plane_yaw, p.translation_plane_pitch = rng.uniform(-0.02, 0.02, 2)
        poses.append(p)
    return poses


@pytest.mark.parametrize("size", [(10, 8), (768, 512), (1024, 768), (7952, 5304), (641, 479)])
def test_roi_matches_oracle(size):
    w, h = size
    rng = np.random.default_rng(w * 7 + h)
    for trial in range(20):
        n = int(rng.integers(1, 6))
        poses = _random_poses(rng, n, w, ("basic", "lens", "trans", "shift"))
        if trial % 3 == 0:
            poses[0] = fsb.ImagePose()
        active = [bool(v) for v in rng.integers(0, 2, n)] if trial % 4 == 1 else [True] * n
        got = fsb.compute_common_overlap_roi(active, [w] * n, [h] * n, poses)
        ref = oracle.compute_roi([p.as_dict() for p in poses], [w] * n, [h] * n, active)
        assert (got.as_tuple() if got else None) == ref


def test_identity_roi_residues_match_reference_chain():
    # the reference's forward chain leaves +-1e-13 residues at identity
    # corners that ceil/floor turn into a one-row ROI change
    for w, h in [(768, 512), (1024, 768), (7952, 5304), (10, 8)]:
        got = fsb.compute_common_overlap_roi([True], [w], [h], [fsb.ImagePose()])
        assert got.as_tuple() == oracle.compute_roi([{}], [w], [h])


@pytest.mark.parametrize("kind", ["basic", "lens", "shift", "trans"])
def test_composed_map_matches_reference_inverse_chain(kind):
    w, h = 1024, 768
    rng = np.random.default_rng({"basic": 1, "lens": 2, "shift": 3, "trans": 4}[kind])
    poses = _random_poses(rng, 6, w, (kind,))
    pts = np.stack([rng.uniform(-20, w + 20, 400), rng.uniform(-20, h + 20, 400)], 1)
    worst = 0.0
    for p in poses:
        got = fsb.inverse_map_points(p, w, h, pts)
        for (x, y), (gx, gy) in zip(pts, got):
            rx, ry = oracle.inverse_point(p.as_dict(), w, h, x, y)
            worst = max(worst, abs(gx - rx), abs(gy - ry))
    assert worst < 1e-8, worst


def test_composed_map_large_frame_and_angles():
    w, h = 7952, 5304
    rng = np.random.default_rng(9)
    pts = np.stack([rng.uniform(0, w, 300), rng.uniform(0, h, 300)], 1)
    for yaw_deg in (0.0, 0.4, 3.0, 15.0):
        p = fsb.ImagePose(yaw=math.radians(yaw_deg), pitch=math.radians(-yaw_deg / 2), roll=math.radians(0.3),
                          hfov_delta=0.1)
        got = fsb.inverse_map_points(p, w, h, pts)
        ref = np.array([oracle.inverse_point(p.as_dict(), w, h, x, y) for x, y in pts])
        assert np.abs(got - ref).max() < 1e-7


# ---- closed forms of the EXPAND used by the kernels, evaluated in numpy f32
def _expand_closed_form(src, dw, dh):
    """Per-output-pixel restatement of the kernels' expand (both modes)."""
    sh, sw = src.shape[:2]
    f32 = np.float32
    exact = max(dw, dh) <= 512
    out = np.zeros((dh, dw, 3), np.float32)

    def s(j, r):
        if exact:
            if j < 0 or j >= sw or r < 0 or r >= sh:
                return np.zeros(3, np.float32)
            return src[r, j]
        return src[min(max(r, 0), sh - 1), min(max(j, 0), sw - 1)]

    def hval(x, r):
        j = x >> 1
        if exact:
            if x % 2 == 0:
                return (s(j - 1, r) + f32(6) * s(j, r)) + s(j + 1, r)
            return f32(4) * (s(j, r) + s(j + 1, r))
        if x % 2 == 0:
            return ((s(j - 1, r) + f32(6) * s(j, r)) + s(j + 1, r)) * f32(0.125)
        return (s(j, r) + s(j + 1, r)) * f32(0.5)

    for y in range(dh):
        q = y >> 1
        for x in range(dw):
            if exact:
                if y % 2 == 0:
                    v = (hval(x, q - 1) + f32(6) * hval(x, q)) + hval(x, q + 1)
                else:
                    v = hval(x, q) + hval(x, q + 1)
                v = v / f32(fsb.exact_expand_divisor(x, y, sw, sh))
            else:
                cq = lambda r: min(max(r, 0), sh - 1)
                if y % 2 == 0:
                    v = ((hval(x, cq(q - 1)) + f32(6) * hval(x, cq(q))) + hval(x, cq(q + 1))) * f32(0.125)
                else:
                    r0 = hval(x, cq(q))
                    v = (r0 + r0) * f32(0.5)
            out[y, x] = v
    return out


@pytest.mark.parametrize("sw,sh", [(1, 1), (1, 3), (3, 1), (2, 2), (2, 5), (5, 2), (4, 4), (7, 5), (6, 9)])
def test_exact_expand_closed_form_is_bitwise_the_reference_skipsm(sw, sh):
    rng = np.random.default_rng(sw * 31 + sh)
    src = rng.uniform(-50, 300, (sh, sw, 3)).astype(np.float32)
    for dw in (2 * sw - 1, 2 * sw):
        for dh in (2 * sh - 1, 2 * sh):
            if dw < 1 or dh < 1:
                continue
            ref = oracle.expand_rgb(src, dw, dh)
            got = _expand_closed_form(src, dw, dh)
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (dw, dh)


@pytest.mark.parametrize("sw,sh,dw,dh", [(257, 3, 513, 5), (260, 4, 519, 8), (3, 300, 6, 599)])
def test_clamped_expand_closed_form_is_bitwise_the_reference(sw, sh, dw, dh):
    rng = np.random.default_rng(sw + sh)
    src = rng.uniform(-50, 300, (sh, sw, 3)).astype(np.float32)
    ref = oracle.expand_rgb(src, dw, dh)
    got = _expand_closed_form(src, dw, dh)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


# ------------------------------------------------------------ serving (host)
def test_stack_footprint_modes_follow_the_budget():
    d = fsb.stack_desc(7952, 5304, 30, fsb.Rect(82, 63, 7872, 5243))
    laps, m_laps, ok = fsb.stack_footprint(d, 1 << 50)
    assert m_laps == "laps" and ok
    fused, m_fused, ok = fsb.stack_footprint(d, laps - 1)
    assert m_fused == "fused" and ok and fused < laps
    cache, m_cache, ok = fsb.stack_footprint(d, fused - 1)
    assert m_cache == "cache" and ok and cache < fused
    resident, m_res, ok = fsb.stack_footprint(d, cache - 1)
    assert m_res == "resident" and ok and resident < cache
    refetch, m_ref, ok = fsb.stack_footprint(d, resident - 1)
    assert m_ref == "refetch" and ok and refetch < resident
    b, _, ok = fsb.stack_footprint(d, refetch - 1)
    assert not ok and b == refetch
    # device-resident frames need no upload staging
    dev_laps, _, _ = fsb.stack_footprint(d, 1 << 50, host_frames=False)
    assert dev_laps < laps
    # FP16 level storage shrinks the level slots
    d16 = fsb.stack_desc(7952, 5304, 30, fsb.Rect(82, 63, 7872, 5243), level_storage=fsb.STORAGE_F16)
    assert fsb.stack_footprint(d16, 1 << 50)[0] < laps


def test_mode_bytes_order():
    d = fsb.stack_desc(7952, 5304, 30, fsb.Rect(82, 63, 7872, 5243))
    b = {m: fsb.stack_mode_bytes(d, m) for m in ("laps", "fused", "cache", "resident", "refetch")}
    assert b["laps"] > b["fused"] > b["cache"] > b["resident"] > b["refetch"]
    # per frame-pixel: laps keeps the f32 level-0 Laplacian (12 B) that fused does not
    n0 = 7872 * 5243 * 30
    assert 11.0 < (b["laps"] - b["fused"]) / n0 < 12.5
    assert fsb.stack_footprint(d, b["cache"])[:2] == (b["cache"], "cache")
    for m in ("laps", "fused"):
        with pytest.raises(fsb.FocusCudaError):  # two levels only: no split pyramid
            fsb.stack_mode_bytes(fsb.stack_desc(2, 1, 2), m)


def test_stack_footprint_rejects_bad_desc():
    with pytest.raises(fsb.FocusCudaError):
        fsb.stack_footprint(fsb.stack_desc(64, 48, 2, contrast_window=4), 1 << 40)


class _FakeCtx:
    def __init__(self):
        self.budget = None
        self.trims = 0

    def set_budget(self, b):
        self.budget = b

    def trim(self):
        self.trims += 1

    def reserve(self, n):
        pass

    def close(self):
        pass


def test_server_admission_respects_the_budget():
    srv = fsb.serving.StackServer(hbm_budget_bytes=80 * 10**9, workers=3, context_factory=_FakeCtx,
                                  max_stack_fraction=1.0)
    big = fsb.serving.StackRequest(0, 0.0, 7952, 5304, 30)
    roi = fsb.Rect(0, 0, 7952, 5304)
    # the server's first mode (the fused split pyramid) fits two stacks
    need = fsb.stack_mode_bytes(fsb.stack_desc(7952, 5304, 30, roi), srv.modes[0])
    w1, b1 = srv._try_admit(big, roi)
    assert b1 == need and w1.busy and w1.ctx.budget == need
    w2, b2 = srv._try_admit(fsb.serving.StackRequest(1, 0.0, 7952, 5304, 30), roi)
    assert w2 is not w1 and b1 + b2 <= srv.budget
    # a third one only fits in a smaller mode or not at all
    third = srv._try_admit(fsb.serving.StackRequest(2, 0.0, 7952, 5304, 30), roi)
    if third is not None:
        assert b1 + b2 + third[1] <= srv.budget
    # idle workers hold no reservation: the shared pool's cached memory is
    # reused, never trimmed by the server (the library trims only when an
    # allocation finds nothing that fits)
    srv2 = fsb.serving.StackServer(hbm_budget_bytes=need + 10**6, workers=2, context_factory=_FakeCtx,
                                   max_stack_fraction=1.0)
    w, b = srv2._try_admit(big, roi)
    assert w is srv2.workers[0] and b == need
    assert all(o.ctx.trims == 0 for o in srv2.workers)


def test_server_caps_one_stacks_share_of_the_budget():
    roi = fsb.Rect(0, 0, 7952, 5304)
    srv = fsb.serving.StackServer(hbm_budget_bytes=40 * 10**9, workers=2, context_factory=_FakeCtx,
                                  max_stack_fraction=0.25)
    w, b = srv._try_admit(fsb.serving.StackRequest(0, 0.0, 7952, 5304, 30), roi)
    assert b <= 10 * 10**9
    assert b < fsb.stack_mode_bytes(fsb.stack_desc(7952, 5304, 30, roi), "cache")


def test_poisson_stream_shape():
    reqs = fsb.serving.poisson_stream(400, 50.0, seed=3)
    assert len(reqs) == 400
    t = [r.arrival_s for r in reqs]
    assert all(b > a for a, b in zip(t, t[1:]))
    assert 4.0 < t[-1] < 12.0  # ~ n / rate
    sizes = {(r.width, r.height) for r in reqs}
    assert sizes <= set(fsb.serving.SIZE_MIX) | {fsb.serving.LARGE}
    assert all(4 <= r.frames <= (143 if (r.width, r.height) == fsb.serving.LARGE else 40) for r in reqs)


@pytest.mark.parametrize("scene,frame", [(0, 0), (0, 5), (1, 3), (1, 29)])
def test_oracle_synthetic_poses_equal_the_library_generator(scene, frame):
    """The CPU legs of bench.py draw poses from the oracle's restatement of
    the generator; they must be the library's poses."""
    got = oracle.synth_pose(1, scene, 7952, 5304, frame, 30)
    want = fsb.synth_pose(1, scene, 7952, 5304, frame, 30).as_dict()
    assert got == want


def test_oracle_synthetic_frame_rows_and_statistics():
    full = oracle.synth_frame(3, oracle.SCENE_SMALL, 320, 240, 2, 8, jobs=4)
    part = oracle.synth_frame(3, oracle.SCENE_SMALL, 320, 240, 2, 8, rows=(100, 20), jobs=3)
    assert np.array_equal(part[100:120], full[100:120])
    assert not part[:100].any() and not part[120:].any()
    assert 90 < full.mean() < 160 and 15 < full.std() < 60


def test_autotuner_caches_the_winner_per_workload(tmp_path, monkeypatch):
    """The batched-form tuner times every candidate once per workload
    signature and answers later calls from its JSON cache (no device work:
    the timing call is replaced by a fake)."""
    from types import SimpleNamespace

    at = fsb.autotune
    calls = []

    def fake_time(ctx, stacks, reps=3, level_storage=0, **knobs):
        calls.append(knobs)
        if knobs["pass2_mode"] == 0:
            raise fsb.FocusCudaError(3, "does not fit")
        return {"knobs": dict(knobs), "s_per_run": 1.0 / knobs["lanes"] + 0.01 * knobs["frames_per_batch"]}

    monkeypatch.setattr(at, "time_batch", fake_time)
    ctx = SimpleNamespace(budget=lambda: 120e9)
    stacks = [SimpleNamespace(width=640, height=480, frames=[0] * 5), SimpleNamespace(width=320, height=240,
                                                                                       frames=[0] * 3)]
    path = str(tmp_path / "tune.json")
    space = {"lanes": (2, 4), "frames_per_batch": (4, 8), "pass2_mode": (3, 0)}
    r1 = at.tune(ctx, stacks, space=space, cache_path=path, schedule_space={})
    assert not r1["cached"] and len(calls) == 8
    assert r1["best"] == {"lanes": 4, "frames_per_batch": 4, "pass2_mode": 3}
    assert sum("skipped" in t for t in r1["trials"]) == 4
    r2 = at.tune(ctx, list(reversed(stacks)), space=space, cache_path=path)
    assert r2["cached"] and r2["best"] == r1["best"] and len(calls) == 8
    # another workload is timed again
    at.tune(ctx, stacks[:1], space=space, cache_path=path, schedule_space={})
    assert len(calls) == 16


def test_autotuner_searches_the_level_schedule_with_the_best_knobs(monkeypatch):
    """After lanes x K x pass-2 mode, the level schedule is timed with the best
    of them (the library's own schedule, all zeros, is not timed twice) and a
    faster schedule becomes part of the winner."""
    from types import SimpleNamespace

    at = fsb.autotune
    calls = []

    def fake_time(ctx, stacks, reps=3, level_storage=0, **knobs):
        calls.append(knobs)
        t = 1.0 / knobs["lanes"] - 0.05 * (knobs.get("fuse_min_tiles", 0) == 296) - 0.01 * (knobs.get("tail_side", 0) == 32)
        return {"knobs": dict(knobs), "s_per_run": t}

    monkeypatch.setattr(at, "time_batch", fake_time)
    ctx = SimpleNamespace(budget=lambda: 120e9)
    stacks = [SimpleNamespace(width=640, height=480, frames=[0] * 5)]
    r = at.tune(ctx, stacks, space={"lanes": (2, 4), "frames_per_batch": (8,), "pass2_mode": (3,)},
                schedule_space={"fuse_min_tiles": (0, 296), "tail_side": (0, 32)})
    assert len(calls) == 2 + 3
    assert all(c["lanes"] == 4 for c in calls[2:])
    assert r["best"] == {"lanes": 4, "frames_per_batch": 8, "pass2_mode": 3, "fuse_min_tiles": 296, "tail_side": 32}
