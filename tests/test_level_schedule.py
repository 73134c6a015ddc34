"""The level schedule of the split-pyramid modes (fs_ctx_set_level_schedule)
changes which kernels run, never the bytes: levels blended together with
their mask REDUCE (the level-0 tile kernel templated on the mask source)
against the two per-level launches, and a shorter or longer small-level
tail, give the same FP32 base bit for bit, in the laps and fused modes and
with FP32 and FP16 level storage."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from __graft_entry__ import load_package  # noqa: E402

fsb = load_package()
pytestmark = pytest.mark.gpu

NEVER = 0xFFFFFFFF
# (fuse_min_tiles, tail_side): the library's defaults, every level >= 1
# fused, none fused, each with the tail limited to sides of 16
SCHEDULES = [(0, 0), (1, 0), (NEVER, 0), (1, 16), (NEVER, 16)]


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return t


def fuse(torch, ctx, frames, poses, W, H, roi, mode, storage):
    st = fsb.PyramidContrastStack(ctx, W, H, len(frames), roi=roi, frames_per_batch=3, level_storage=storage,
                                  pass2_mode=mode)
    assert st.pass2_mode == mode
    base = torch.zeros((roi.height, roi.width, 3), dtype=torch.float32, device="cuda:0")
    st.set_base_output(base, roi.width * 3)
    for f, p in zip(frames, poses):
        st.add_frame(f, p)
    out = st.finish()
    st.close()
    return out, base.cpu().numpy()


@pytest.mark.parametrize("storage", [fsb.STORAGE_F32, fsb.STORAGE_F16])
@pytest.mark.parametrize("mode", ["laps", "fused"])
def test_level_schedules_give_identical_bytes(torch, mode, storage):
    W, H, F = 1100, 820, 5
    with fsb.Context(0) as ctx:
        frames, poses = [], []
        for k in range(F):
            buf = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda:0")
            poses.append(fsb.synth_frame_device(ctx, 31, fsb.SCENE_SMALL, W, H, k, F, buf, W * 3))
            frames.append(buf.cpu().numpy())
        roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
        ref = None
        for fuse_min_tiles, tail_side in SCHEDULES:
            ctx.set_level_schedule(fuse_min_tiles, tail_side)
            out, base = fuse(torch, ctx, frames, poses, W, H, roi, mode, storage)
            if ref is None:
                ref = (out, base)
                continue
            assert np.array_equal(out, ref[0]), (fuse_min_tiles, tail_side)
            assert np.array_equal(base.view(np.uint32), ref[1].view(np.uint32)), (fuse_min_tiles, tail_side)


def test_level_schedule_rejects_a_tail_beyond_the_tail_kernels(torch):
    with fsb.Context(0) as ctx:
        with pytest.raises(fsb.FocusCudaError) as e:
            ctx.set_level_schedule(0, 65)
        assert e.value.code == "FS_ERR_INVALID"
        ctx.set_level_schedule(0, 64)
