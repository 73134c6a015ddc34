"""16-bit samples (the reference's u16 twins) through the C ABI, against the
CPU oracle's u16 path.

Bar: remap alpha bit-exact everywhere and RGB bit-exact wherever alpha > 0
(src/remap.zig:841-937); fused output within one LSB of the 16-bit output
(|base_gpu - base_oracle| <= 1 in 16-bit units, u16 output within 1), the
reference's own "<= 1 LSB on 16-bit" bar read on a native 16-bit image.
"""
import numpy as np
import pytest

import oracle
from __graft_entry__ import load_package

fsb = load_package()

FS_ERR_UNSUPPORTED = 8


def to_u16(frames, seed):
    """16-bit frames with the 8-bit frames' structure and random low bits."""
    rng = np.random.default_rng(seed)
    return [(f.astype(np.uint16) * 257 + rng.integers(0, 257, f.shape, dtype=np.uint16)).astype(np.uint16)
            for f in frames]


def test_desc_checks_for_16_bit_stacks():
    # argument checks only: no GPU needed
    d = fsb.stack_desc(640, 480, 20, sample_bits=16)
    assert fsb.stack_mode_bytes(d, "resident") > fsb.stack_mode_bytes(d, "refetch")
    for mode in ("cache", "laps", "fused"):
        with pytest.raises(fsb.FocusCudaError):
            fsb.stack_mode_bytes(d, mode)
    with pytest.raises(fsb.FocusCudaError) as e:
        fsb.stack_mode_bytes(fsb.stack_desc(640, 480, 4, sample_bits=16, level_storage=fsb.STORAGE_F16), "resident")
    assert e.value.code == "FS_ERR_UNSUPPORTED"
    with pytest.raises(fsb.FocusCudaError):
        fsb.stack_mode_bytes(fsb.stack_desc(640, 480, 4, sample_bits=12), "resident")


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


def synth16(torch, ctx, W, H, F, seed):
    frames, poses = [], []
    for k in range(F):
        buf = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda:0")
        poses.append(fsb.synth_frame_device(ctx, seed, fsb.SCENE_SMALL, W, H, k, F, buf, W * 3))
        frames.append(buf.cpu().numpy())
    return to_u16(frames, seed), poses


def assert_remap16_equal(got, ref):
    ch = got.shape[2] - 1
    assert np.array_equal(got[..., ch], ref[..., ch]), int((got[..., ch] != ref[..., ch]).sum())
    vis = ref[..., ch] > 0
    assert np.array_equal(got[vis], ref[vis]), int((got[vis] != ref[vis]).any(-1).sum())


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["basic", "lens"])
def test_remap16_bit_exact(torch, ctx, kind):
    W, H = 400, 300
    frames, poses = synth16(torch, ctx, W, H, 3, seed=5)
    rng = np.random.default_rng(3)
    for f, p in zip(frames, poses):
        pose = fsb.ImagePose(**p.as_dict())
        if kind == "lens":
            pose.radial_a, pose.radial_b, pose.radial_c = rng.uniform(-0.01, 0.01, 3)
        roi = fsb.Rect(-7, 5, W - 20, H + 9)
        got = fsb.remap_rigid_image(ctx, f, pose, roi)
        ref = oracle.remap(f, pose.as_dict(), roi.as_tuple())
        assert got.dtype == np.uint16
        assert_remap16_equal(got, ref)
    gray = np.ascontiguousarray(frames[0][..., 1])
    got = fsb.remap_rigid_image(ctx, gray, poses[1])
    assert_remap16_equal(got, oracle.remap(gray, poses[1].as_dict(), None))


def check16(out, base, ref_out, ref_base):
    d = np.abs(base - ref_base)
    assert d.max() <= 1.0, f"max |base diff| = {d.max()} LSB of 16 bits"
    du = np.abs(out.astype(np.int64) - ref_out.astype(np.int64))
    assert du.max() <= 1


def fuse16(torch, ctx, frames, poses, roi, mode=None, aligned=False):
    h, w, c = frames[0].shape
    st = fsb.PyramidContrastStack(ctx, w, h, len(frames), roi=None if aligned else roi, channels=c, aligned=aligned,
                                  sample_bits=16, pass2_mode=mode, frames_per_batch=3)
    if mode:
        assert st.pass2_mode == mode
    base = torch.zeros((st.out_height, st.out_width, 3), dtype=torch.float32, device="cuda:0")
    st.set_base_output(base, st.out_width * 3)
    for f, p in zip(frames, poses):
        st.add_frame(f, p)
    out = st.finish(refetch=lambda i: frames[i])
    st.close()
    assert out.dtype == np.uint16
    return out, base.cpu().numpy().astype(np.float64)


@pytest.mark.gpu
@pytest.mark.parametrize("W,H,F,mode", [(320, 240, 5, "resident"), (640, 480, 4, "refetch"), (1100, 700, 3, None),
                                        (7, 5, 2, None)])
def test_stack_fusion16_matches_oracle(torch, ctx, W, H, F, mode):
    frames, poses = synth16(torch, ctx, W, H, F, seed=W + H)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses) or fsb.Rect(0, 0, W, H)
    out, base = fuse16(torch, ctx, frames, poses, roi, mode)
    ref_out, ref_base = oracle.stack_fuse(frames, [p.as_dict() for p in poses], roi.as_tuple(), jobs=8,
                                          want_base=True)
    check16(out, base, ref_out, ref_base)


@pytest.mark.gpu
def test_aligned_rgba16_fusion_matches_oracle(torch, ctx):
    W, H, F = 256, 192, 4
    frames, poses = synth16(torch, ctx, W, H, F, seed=9)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
    aligned = [oracle.remap(f, p.as_dict(), roi.as_tuple()) for f, p in zip(frames, poses)]
    out, base = fuse16(torch, ctx, aligned, [None] * F, None, aligned=True)
    ref_out, ref_base = oracle.fuse_aligned(aligned, want_base=True)
    check16(out, base, ref_out, ref_base)


@pytest.mark.gpu
def test_single_pixel_stack16(torch, ctx):
    frames = [np.full((1, 1, 3), v, np.uint16) for v in (1000, 50000, 30000)]
    out, base = fuse16(torch, ctx, frames, [None] * 3, None, aligned=True)
    ref_out, ref_base = oracle.fuse_aligned(frames, want_base=True)
    check16(out, base, ref_out, ref_base)
