"""hybrid-pyramid-contrast through the C ABI (fs_stack_set_method), against
the oracle's restatement of the reference's hybrid branch
(src/stack/pipeline.zig:177-236, src/fuse/blend.zig:188-289,
src/fuse/pyramid.zig:271-301, 418-488).

The hybrid image is a function of two 8-bit images, the pyramid-contrast
("soft") output and the hardmask-contrast ("hard") winners' colours:
  * the merge is compared with the oracle's merge of the library's own soft
    and hard images (same inputs: the plain REDUCE, EXPAND, Laplacian, mix
    and collapse must agree to FP32 rounding, u8 within 1);
  * the winners are compared with the oracle's: identical wherever the two
    largest weights of a pixel are not within FP32 rounding of each other
    (the library's contrast weights agree with the reference's to ~1e-7
    relative, so a near-tie may pick the other frame);
  * end to end the image is within 2 u8 steps of the oracle's (its soft
    input is within 1).
"""
import numpy as np
import pytest

import oracle
from __graft_entry__ import load_package

fsb = load_package()
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


@pytest.fixture(scope="module")
def ctx(torch):
    c = fsb.Context(0)
    yield c
    c.close()


def synth(torch, ctx, W, H, F, seed):
    frames, poses = [], []
    for k in range(F):
        buf = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda:0")
        poses.append(fsb.synth_frame_device(ctx, seed, fsb.SCENE_SMALL, W, H, k, F, buf, W * 3))
        frames.append(buf.cpu().numpy())
    return frames, poses


def run(torch, ctx, frames, poses, roi, method, mode, sharpness=0.35):
    H, W = frames[0].shape[:2]
    st = fsb.PyramidContrastStack(ctx, W, H, len(frames), roi=roi, method=method, hybrid_sharpness=sharpness,
                                  pass2_mode=mode, frames_per_batch=3)
    assert st.pass2_mode == mode
    base = torch.zeros((roi.height, roi.width, 3), dtype=torch.float32, device="cuda:0")
    st.set_base_output(base, roi.width * 3)
    for f, p in zip(frames, poses):
        st.add_frame(f, p)
    out = st.finish(refetch=lambda i: frames[i])
    hard = None
    if method != "pyramid-contrast":
        buf = torch.as_tensor(st.buffer(fsb.BUFFER_HARD), device="cuda:0")
        words = buf[:roi.height, :roi.width].cpu().numpy().view(np.uint32)
        hard = np.stack([(words >> (8 * c)) & 255 for c in range(3)], axis=-1).astype(np.uint8)
    st.close()
    return out, base.cpu().numpy().astype(np.float64), hard


@pytest.fixture(scope="module")
def stack(torch, ctx):
    W, H, F = 640, 480, 6
    frames, poses = synth(torch, ctx, W, H, F, seed=17)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
    ref_out, ref_base, ref_hard = oracle.stack_fuse_hybrid(frames, [p.as_dict() for p in poses], roi.as_tuple(),
                                                           jobs=8, want_base=True, want_hard=True)
    return frames, poses, roi, ref_out, ref_base, ref_hard


@pytest.mark.parametrize("mode", ["laps", "fused", "cache", "resident"])
def test_hybrid_matches_oracle(torch, ctx, stack, mode):
    frames, poses, roi, ref_out, ref_base, ref_hard = stack
    soft, _, _ = run(torch, ctx, frames, poses, roi, "pyramid-contrast", mode)
    out, base, hard = run(torch, ctx, frames, poses, roi, "hybrid-pyramid-contrast", mode)
    # the merge, on the library's own soft and hard images
    m_out, m_base = oracle.hybrid_merge(soft, hard, jobs=8)
    assert np.abs(base - m_base).max() <= 1e-3
    assert np.abs(out.astype(np.int16) - m_out.astype(np.int16)).max() <= 1
    # the winners: identical but for near-ties of the two largest weights
    differ = (hard != ref_hard).any(-1)
    assert differ.mean() <= 1e-4, int(differ.sum())
    # end to end
    assert np.abs(out.astype(np.int16) - ref_out.astype(np.int16)).max() <= 2
    assert np.mean(np.abs(base - ref_base) <= 1.0) >= 0.9999


def test_hybrid_sharpness_zero_reconstructs_the_soft_image(torch, ctx, stack):
    frames, poses, roi = stack[:3]
    soft, _, _ = run(torch, ctx, frames, poses, roi, "pyramid-contrast", "laps")
    out, _, _ = run(torch, ctx, frames, poses, roi, "hybrid-pyramid-contrast", "laps", sharpness=0.0)
    assert np.abs(out.astype(np.int16) - soft.astype(np.int16)).max() <= 1


def test_hybrid_method_errors(torch, ctx):
    with pytest.raises(fsb.FocusCudaError) as e:
        fsb.PyramidContrastStack(ctx, 64, 48, 2, method="hybrid-pyramid-contrast", hybrid_sharpness=1.5)
    assert e.value.code == "FS_ERR_INVALID"
    with pytest.raises(fsb.FocusCudaError) as e:
        fsb.PyramidContrastStack(ctx, 64, 48, 2, method="hybrid-pyramid-contrast", sample_bits=16)
    assert e.value.code == "FS_ERR_UNSUPPORTED"
    st = fsb.PyramidContrastStack(ctx, 64, 48, 2, method="hybrid-pyramid-contrast", aligned=True)
    with pytest.raises(fsb.FocusCudaError) as e:
        st.set_frame_total(4)
    assert e.value.code == "FS_ERR_UNSUPPORTED"
    st.close()
