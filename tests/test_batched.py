"""Batched form on the device: several stacks of mixed sizes fused by one
StackBatch (direct run, then a captured CUDA graph replayed) must give the
same bytes as fusing each stack alone, in FP32 and in FP16 level storage, and
a replay after the frames were refilled in place must follow the new frames."""
import numpy as np
import pytest

from __graft_entry__ import load_package

fsb = load_package()
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def make_stacks(torch, ctx, specs, seed):
    stacks = []
    for j, (w, h, n) in enumerate(specs):
        frames, poses = [], []
        for k in range(n):
            buf = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda:0")
            poses.append(fsb.synth_frame_device(ctx, seed + j, fsb.SCENE_SMALL, w, h, k, n, buf, w * 3))
            frames.append(buf)
        roi = fsb.compute_common_overlap_roi([True] * n, [w] * n, [h] * n, poses)
        out = torch.zeros((roi.height, roi.width, 3), dtype=torch.uint8, device="cuda:0")
        stacks.append(fsb.BatchStack(frames, poses, roi, out, w, h))
    return stacks


def alone(torch, ctx, st, storage, k=0, mode="cache"):
    # the cache / resident / laps modes give the same bytes; the fused mode
    # blends level 0 in another rounding order, so it is compared with itself
    s = fsb.PyramidContrastStack(ctx, st.width, st.height, len(st.frames), roi=st.roi, level_storage=storage,
                                 frames_per_batch=k, pass2_mode=mode)
    for f, p in zip(st.frames, st.poses):
        s.add_frame_device(f, st.width * 3, p)
    out = s.finish()
    s.close()
    return out


@pytest.mark.parametrize("storage", [fsb.STORAGE_F32, fsb.STORAGE_F16])
@pytest.mark.parametrize("pass2_mode", [0, 1, 3, 4])
def test_batch_matches_stacks_alone(torch, storage, pass2_mode):
    """Every stack of the batch gives the bytes of the same stack fused alone
    in the same pass-2 mode, on the direct run and on graph replays, with
    the stacks of a lane sharing one arena."""
    ctx = fsb.Context(0)
    specs = [(320, 240, 5), (640, 480, 9), (200, 150, 3), (512, 384, 12), (320, 240, 4)]
    stacks = make_stacks(torch, ctx, specs, seed=40)
    name = fsb.api.PASS2_MODES[pass2_mode]
    want = [alone(torch, ctx, st, storage, mode=name) for st in stacks]
    with fsb.StackBatch(ctx, stacks, lanes=3, pass2_mode=pass2_mode, level_storage=storage) as b:
        assert b.pass2_modes() == [name] * len(stacks)
        for run in range(3):
            for st in stacks:
                st.out.zero_()
            b.run()
            assert b.uses_graph == (run >= 1)
            for st, w in zip(stacks, want):
                assert np.array_equal(st.out.cpu().numpy(), w), (run, st.width, st.height)
    ctx.close()


def test_replay_reads_refilled_frames(torch):
    ctx = fsb.Context(0)
    specs = [(320, 240, 4), (256, 192, 6)]
    stacks = make_stacks(torch, ctx, specs, seed=60)
    with fsb.StackBatch(ctx, stacks, lanes=2) as b:
        b.run()
        b.run()
        # new content at the same addresses: frames of another scene seed
        for j, st in enumerate(stacks):
            n = len(st.frames)
            for k, f in enumerate(st.frames):
                fsb.synth_frame_device(ctx, 99 + j, fsb.SCENE_SMALL, st.width, st.height, k, n, f, st.width * 3)
        ctx.synchronize()
        b.run()
        assert b.uses_graph
        for st in stacks:
            assert np.array_equal(st.out.cpu().numpy(), alone(torch, ctx, st, fsb.STORAGE_F32))
    ctx.close()


def test_autotuner_picks_a_fitting_candidate(torch):
    ctx = fsb.Context(0)
    stacks = make_stacks(torch, ctx, [(320, 240, 5), (640, 480, 6), (256, 192, 3)], seed=70)
    res = fsb.autotune.tune(ctx, stacks, space={"lanes": (1, 3), "frames_per_batch": (4, 8), "pass2_mode": (0,)},
                            reps=2)
    assert res["best"] in [t["knobs"] for t in res["trials"]]
    assert all(t.get("graph", True) for t in res["trials"])
    ctx.close()


def test_lanes_share_their_arena(torch):
    """A batch holds about one arena per lane (its largest stack), not the sum
    over its stacks: four equal stacks on two lanes hold about half of what
    four stacks alone would, and the default mode takes the split pyramid."""
    ctx = fsb.Context(0)
    stacks = make_stacks(torch, ctx, [(640, 480, 6)] * 4, seed=80)
    one = fsb.api.stack_mode_bytes(fsb.api.stack_desc(640, 480, 6, stacks[0].roi), "laps", host_frames=False)
    before = ctx.device_bytes()
    with fsb.StackBatch(ctx, stacks, lanes=2) as b:
        assert b.pass2_modes() == ["laps"] * 4
        held = ctx.device_bytes() - before
        assert 2 * one <= held < 3 * one, (held, one)
        b.run()
        b.run()
        for st in stacks:
            assert np.array_equal(st.out.cpu().numpy(), alone(torch, ctx, st, fsb.STORAGE_F32, mode="laps"))
    assert ctx.device_bytes() == before
    ctx.close()
