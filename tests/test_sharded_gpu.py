"""Frame-sharded stack through the library's phase entry points on one GPU:
two shards of one stack, their weight sums summed and unions maxed between
pass 1 and pass 2 and their accumulators summed before the collapse (what
fuse_sharded does with collectives across GPUs), against the same stack
fused whole.  The only difference is the order of FP32 sums."""
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


@pytest.mark.parametrize("mode", ["laps", "cache"])
def test_two_shards_match_the_whole_stack(torch, mode):
    W, H, F = 640, 480, 7
    ctx = fsb.Context(0)
    frames, poses = [], []
    for k in range(F):
        buf = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda:0")
        poses.append(fsb.synth_frame_device(ctx, 3, fsb.SCENE_SMALL, W, H, k, F, buf, W * 3))
        frames.append(buf)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)

    def make(lo, hi):
        st = fsb.PyramidContrastStack(ctx, W, H, hi - lo, roi=roi, frames_per_batch=3, pass2_mode=mode)
        base = torch.zeros((st.out_height, st.out_width, 3), dtype=torch.float32, device="cuda:0")
        st.set_base_output(base, st.out_width * 3)
        for k in range(lo, hi):
            st.add_frame_device(frames[k], W * 3, poses[k])
        return st, base

    whole, whole_base = make(0, F)
    want = whole.finish()
    whole.close()

    shards = [make(*fsb.sharded.shard_range(F, 2, r)) for r in range(2)]
    for st, _ in shards:
        st.set_frame_total(F)
        st.end_pass1()
    norms = [torch.as_tensor(st.buffer(fsb.BUFFER_WEIGHT_SUM), device="cuda:0") for st, _ in shards]
    unis = [torch.as_tensor(st.buffer(fsb.BUFFER_UNION), device="cuda:0") for st, _ in shards]
    total, union = norms[0] + norms[1], torch.maximum(unis[0], unis[1])
    for n, u in zip(norms, unis):
        n.copy_(total)
        u.copy_(union)
    torch.cuda.synchronize()
    for st, _ in shards:
        st.blend()
    levels = fsb.sharded.level_count(shards[0][0].out_width, shards[0][0].out_height)
    for lvl in range(levels):
        a = torch.as_tensor(shards[0][0].buffer(fsb.BUFFER_ACCUMULATOR, lvl), device="cuda:0")
        b = torch.as_tensor(shards[1][0].buffer(fsb.BUFFER_ACCUMULATOR, lvl), device="cuda:0")
        a += b
    torch.cuda.synchronize()
    got = shards[0][0].collapse()
    with pytest.raises(fsb.FocusCudaError):  # phases run once, in order
        shards[1][0].end_pass1()
    d = np.abs(shards[0][1].cpu().numpy().astype(np.float64) - whole_base.cpu().numpy().astype(np.float64))
    assert d.max() <= 1e-3, d.max()
    assert np.abs(got.astype(np.int16) - want.astype(np.int16)).max() <= 1
    for st, _ in shards:
        st.close()
    ctx.close()
