"""GPU parity: libfocuscuda (through its C ABI) against the CPU oracle.

Bar: remap alpha bit-exact everywhere and RGB bit-exact wherever alpha > 0;
fused output within 1 LSB of the 16-bit grid (|base_gpu - base_oracle| <=
1/257 in 8-bit units) of the oracle's FP32 evaluation, and u8 output within
1 LSB.

RGB of alpha-0 pixels: a sample that lands within ~1e-13 px of the integer
one pixel outside the frame (identity-like poses put it exactly there) gets
RGB = the edge pixel when the reference's rounding residue is positive and 0
when it is negative (src/remap.zig:736-752), with alpha 0 either way.  That
residue comes from the last bit of the reference's trig chain, so those
invisible samples are compared separately and only bounded in count.
"""
import math

import numpy as np
import pytest

import oracle
from __graft_entry__ import load_package

fsb = load_package()
pytestmark = pytest.mark.gpu

LSB16 = 1.0 / 257.0


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


def synth_stack(torch, ctx, W, H, F, seed, scene=fsb.SCENE_SMALL):
    frames, poses = [], []
    for k in range(F):
        buf = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda:0")
        poses.append(fsb.synth_frame_device(ctx, seed, scene, W, H, k, F, buf, W * 3))
        frames.append(buf.cpu().numpy())
    return frames, poses


def gpu_fuse(ctx, torch, frames, poses, roi, window=5, k=0, aligned=False):
    h, w = frames[0].shape[:2]
    c = frames[0].shape[2]
    st = fsb.PyramidContrastStack(ctx, w, h, len(frames), roi=None if aligned else roi, channels=c,
                                  contrast_window=window, aligned=aligned, frames_per_batch=k)
    base = torch.zeros((st.out_height, st.out_width, 3), dtype=torch.float32, device="cuda:0")
    st.set_base_output(base, st.out_width * 3)
    for f, p in zip(frames, poses):
        st.add_frame(f, p)
    out = st.finish()
    st.close()
    return out, base.cpu().numpy().astype(np.float64)


def with_kind(pose, kind, rng):
    p = fsb.ImagePose(**pose.as_dict())
    if kind == "lens":
        p.radial_a, p.radial_b, p.radial_c = rng.uniform(-0.01, 0.01, 3)
        p.center_shift_x, p.center_shift_y = rng.uniform(-2, 2, 2)
    elif kind == "shift":
        p.center_shift_x, p.center_shift_y = rng.uniform(-2, 2, 2)
    elif kind == "trans":
        p.trans_x, p.trans_y, p.trans_z = rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(-0.01, 0.01)
        p.translation_plane_yaw, p.translation_plane_pitch = rng.uniform(-0.01, 0.01, 2)
    return p


# ------------------------------------------------------------------ remap
def test_identity_remap_preserves_interior_grayscale_pixels(ctx):
    # src/remap.zig:1018-1057 through the GPU
    src = np.arange(1, 26, dtype=np.uint8).reshape(5, 5)
    out = fsb.remap_rigid_image(ctx, src, fsb.ImagePose())
    assert out.shape == (5, 5, 2)
    assert (out[2, 2, 0], out[2, 2, 1]) == (13, 255)
    assert (out[3, 2, 0], out[3, 2, 1]) == (18, 255)
    assert (out[2, 3, 0], out[2, 3, 1]) == (14, 255)
    assert np.array_equal(out, oracle.remap(src, {}, None))


def assert_remap_equal(got, ref, max_alpha0_rgb=None):
    assert got.shape == ref.shape
    ch = got.shape[2] - 1
    assert np.array_equal(got[..., ch], ref[..., ch]), int((got[..., ch] != ref[..., ch]).sum())
    vis = ref[..., ch] > 0
    assert np.array_equal(got[vis], ref[vis]), int((got[vis] != ref[vis]).any(-1).sum())
    hidden = int((got[~vis] != ref[~vis]).any(-1).sum())
    if max_alpha0_rgb is not None:
        assert hidden <= max_alpha0_rgb, hidden
    return hidden


def _full(band, rows, h):
    full = np.zeros((h,) + band.shape[1:], band.dtype)
    full[rows[0]:rows[1]] = band
    return full


def test_identity_remap_matches_reference_golden_tiff(ctx, golden):
    h, w = int(golden["height"]), int(golden["width"])
    rows = golden["ident_rows"]
    src = _full(golden["ident_src"], rows, h)
    out = fsb.remap_rigid_image(ctx, src, fsb.ImagePose(), fsb.Rect(0, int(rows[0]), w, int(rows[1])))
    assert np.array_equal(out, golden["ident_golden"])


def test_pair_pose_remap_matches_oracle_and_golden(ctx, golden):
    h, w = int(golden["height"]), int(golden["width"])
    yaw, pitch, roll, dv, base = golden["pose_values"]
    pose = fsb.ImagePose(yaw=yaw, pitch=pitch, roll=roll, hfov_delta=dv, base_hfov_degrees=base)
    src = _full(golden["pose_src"], golden["pose_src_rows"], h)
    r0, r1 = (int(v) for v in golden["pose_out_rows"])
    out = fsb.remap_rigid_image(ctx, src, pose, fsb.Rect(0, r0, w, r1))
    assert np.array_equal(out, oracle.remap(src, pose.as_dict(), (0, r0, w, r1)))
    ref = golden["pose_golden"]
    m = (out[..., 3] == 255) & (ref[..., 3] == 255)
    d = (out[..., :3].astype(np.float64) - ref[..., :3])[m]
    assert math.sqrt((d ** 2).mean()) / 255.0 <= 0.005


@pytest.mark.parametrize("kind", ["basic", "shift", "lens", "trans"])
@pytest.mark.parametrize("size", [(320, 240), (97, 61)])
def test_remap_bit_exact(torch, ctx, kind, size):
    W, H = size
    frames, poses = synth_stack(torch, ctx, W, H, 4, seed=11)
    rng = np.random.default_rng(5)
    for k in range(4):
        pose = with_kind(poses[k], kind, rng)
        for roi in (None, fsb.Rect(3, 2, W - 5, H - 1), fsb.Rect(-4, -3, W + 6, H + 2)):
            got = fsb.remap_rigid_image(ctx, frames[k], pose, roi)
            ref = oracle.remap(frames[k], pose.as_dict(), roi.as_tuple() if roi else None)
            # alpha-0 RGB can differ only on the one-pixel ring just outside the frame
            assert_remap_equal(got, ref, max_alpha0_rgb=2 * (W + H) + 8)


def test_remap_bit_exact_production_frame(torch, ctx):
    # a full 7952x5304 frame of the production scene (shifts up to 60 px, roll 0.3 deg)
    W, H = 7952, 5304
    buf = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda:0")
    pose = fsb.synth_frame_device(ctx, 3, fsb.SCENE_PRODUCTION, W, H, 5, 30, buf, W * 3)
    src = buf.cpu().numpy()
    roi = fsb.Rect(61, 57, W - 64, H - 70)
    got = fsb.remap_rigid_image(ctx, src, pose, roi)
    ref = oracle.remap(src, pose.as_dict(), roi.as_tuple(), jobs=8)
    assert np.array_equal(got, ref), int((got != ref).any(-1).sum())
    gray = np.ascontiguousarray(src[..., 1])
    groi = fsb.Rect(-30, -20, W + 25, H + 40)
    g = fsb.remap_rigid_image(ctx, gray, pose, groi)
    assert_remap_equal(g, oracle.remap(gray, pose.as_dict(), groi.as_tuple(), jobs=8), max_alpha0_rgb=0)


# ----------------------------------------------------------------- fusion
def check_fused(out, base, ref_out, ref_base):
    d = np.abs(base - ref_base)
    assert d.max() <= LSB16, f"max |base diff| = {d.max()} > 1/257"
    du = np.abs(out.astype(np.int32) - ref_out.astype(np.int32))
    assert du.max() <= 1


@pytest.mark.parametrize("W,H,F,window", [
    (320, 240, 4, 5), (513, 511, 3, 5), (64, 48, 3, 3), (200, 150, 5, 7), (130, 70, 9, 5),
    (7, 5, 2, 3), (2, 3, 2, 3), (1, 1, 2, 3), (4, 9, 3, 5),
])
def test_stack_fusion_matches_oracle(torch, ctx, W, H, F, window):
    frames, poses = synth_stack(torch, ctx, W, H, F, seed=W * 100 + H)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses) or fsb.Rect(0, 0, W, H)
    out, base = gpu_fuse(ctx, torch, frames, poses, roi, window)
    ref_out, ref_base = oracle.stack_fuse(frames, [p.as_dict() for p in poses], roi.as_tuple(), window=window,
                                          want_base=True)
    check_fused(out, base, ref_out, ref_base)


def test_config0_stack_matches_oracle(torch, ctx):
    # 8 RGB frames of 1024x768, small scene, default levels, FP32
    W, H, F = 1024, 768, 8
    frames, poses = synth_stack(torch, ctx, W, H, F, seed=0)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
    assert roi is not None and roi.as_tuple() == oracle.compute_roi([p.as_dict() for p in poses], [W] * F, [H] * F)
    out, base = gpu_fuse(ctx, torch, frames, poses, roi)
    ref_out, ref_base = oracle.stack_fuse(frames, [p.as_dict() for p in poses], roi.as_tuple(), jobs=8,
                                          want_base=True)
    check_fused(out, base, ref_out, ref_base)
    _, ref64 = oracle.stack_fuse(frames, [p.as_dict() for p in poses], roi.as_tuple(), jobs=8, precision=64,
                                 want_base=True)
    assert np.abs(base - ref64).max() <= LSB16


@pytest.mark.parametrize("channels", [3, 4])
def test_aligned_fusion_matches_oracle(torch, ctx, channels):
    W, H, F = 256, 192, 5
    frames, poses = synth_stack(torch, ctx, W, H, F, seed=21)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
    aligned = [oracle.remap(f, p.as_dict(), roi.as_tuple()) for f, p in zip(frames, poses)]
    if channels == 3:
        aligned = [np.ascontiguousarray(a[..., :3]) for a in aligned]
    out, base = gpu_fuse(ctx, torch, aligned, [None] * F, None, aligned=True)
    ref_out, ref_base = oracle.fuse_aligned(aligned, want_base=True)
    check_fused(out, base, ref_out, ref_base)


def test_batch_size_does_not_change_results(torch, ctx):
    W, H, F = 300, 200, 7
    frames, poses = synth_stack(torch, ctx, W, H, F, seed=4)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
    outs = [gpu_fuse(ctx, torch, frames, poses, roi, k=k) for k in (1, 3, 8)]
    for o, b in outs[1:]:
        assert np.array_equal(o, outs[0][0])
        assert np.array_equal(b, outs[0][1])


def test_identical_frames_fuse_to_the_frame(torch, ctx):
    # size-independent property: with identity poses, fusing copies of one
    # frame reconstructs it (masks sum to one on every level)
    W, H = 7952, 5304
    buf = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda:0")
    fsb.synth_frame_device(ctx, 1, fsb.SCENE_PRODUCTION, W, H, 0, 30, buf, W * 3)
    st = fsb.PyramidContrastStack(ctx, W, H, 3, roi=None, frames_per_batch=3)
    for _ in range(3):
        st.add_frame_device(buf, W * 3, fsb.ImagePose())
    out = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda:0")
    st.finish_device(out, W * 3)
    st.close()
    d = (out.int() - buf.int()).abs()
    assert int(d.max()) <= 1
    assert float((d > 0).float().mean()) < 1e-4


def test_refetch_path_matches_resident(torch, ctx):
    W, H, F = 200, 120, 5
    frames, poses = synth_stack(torch, ctx, W, H, F, seed=8)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
    ref, _ = gpu_fuse(ctx, torch, frames, poses, roi, k=2)
    # a budget that fits the stack in the refetch mode only
    b = fsb.stack_footprint(fsb.stack_desc(W, H, F, roi, frames_per_batch=2), 1 << 50)[0]
    while True:
        b2, mode, ok = fsb.stack_footprint(fsb.stack_desc(W, H, F, roi, frames_per_batch=2), b - 1)
        if not ok:
            break
        b = b2
        if mode == "refetch":
            break
    small = fsb.Context(0, hbm_budget_bytes=b)
    st = fsb.PyramidContrastStack(small, W, H, F, roi=roi, frames_per_batch=2)
    assert st.pass2_mode == "refetch"
    for f, p in zip(frames, poses):
        st.add_frame(f, p)
    calls = []

    def refetch(i):
        calls.append(i)
        return frames[i]

    out = st.finish(refetch=refetch)
    st.close()
    small.close()
    assert calls == list(range(F))
    assert np.array_equal(out, ref)


def close_outputs(a, b):
    d = np.abs(a.astype(np.int16) - b.astype(np.int16))
    return int(d.max()) <= 1 and float((d > 0).mean()) < 1e-3


def test_pass2_modes_give_identical_results(torch, ctx):
    # cache (pass-1 planes kept), resident (frames kept, remapped again) and
    # refetch (frames fetched again) must produce the same bytes; laps (pass 1
    # builds the pyramids) and fused (pass 1 also blends level 0 as
    # sum(lap * w) / N) round level 0 in another order: within one u8 step of
    # them, on a handful of pixels at most.  Each budget is the footprint of
    # its mode, the largest the stack picks there
    W, H, F = 240, 160, 8
    frames, poses = synth_stack(torch, ctx, W, H, F, seed=12)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
    d = fsb.stack_desc(W, H, F, roi, frames_per_batch=3)
    budgets = {}
    avail = 1 << 50
    while True:
        b, mode, ok = fsb.stack_footprint(d, avail)
        if not ok:
            break
        budgets.setdefault(mode, b)
        avail = b - 1
    assert set(budgets) == {"laps", "fused", "cache", "resident", "refetch"}
    results = {}
    for want, budget in budgets.items():
        c = fsb.Context(0, hbm_budget_bytes=budget)
        st = fsb.PyramidContrastStack(c, W, H, F, roi=roi, frames_per_batch=3)
        assert st.pass2_mode == want
        for f, p in zip(frames, poses):
            st.add_frame(f, p)
        results[want] = st.finish(refetch=lambda i: frames[i])
        st.close()
        c.close()
    for m in ("resident", "refetch"):
        assert np.array_equal(results["cache"], results[m]), m
    for m in ("laps", "fused"):
        assert close_outputs(results[m], results["cache"]), m

@pytest.mark.parametrize("mode", ["laps", "fused"])
@pytest.mark.parametrize("storage", [fsb.STORAGE_F32, fsb.STORAGE_F16])
@pytest.mark.parametrize("W,H,F", [(320, 240, 5), (130, 70, 9), (1100, 700, 3)])
def test_small_level_tail_matches_per_level_launches(torch, ctx, mode, storage, W, H, F):
    """finish() blends the split pyramid's small levels (sides <= 64) and
    collapses them in the tail launches; the phase entry points (end_pass1,
    blend, collapse) launch those levels one by one.  Same operations in the
    same order: the same output bytes and collapsed base."""
    frames, poses = synth_stack(torch, ctx, W, H, F, seed=W + F)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
    outs = []
    for phases in (False, True):
        st = fsb.PyramidContrastStack(ctx, W, H, F, roi=roi, frames_per_batch=3, pass2_mode=mode,
                                      level_storage=storage)
        base = torch.zeros((roi.height, roi.width, 3), dtype=torch.float32, device="cuda:0")
        st.set_base_output(base, roi.width * 3)
        for f, p in zip(frames, poses):
            st.add_frame(f, p)
        if phases:
            st.end_pass1()
            st.blend()
            out = st.collapse()
        else:
            out = st.finish()
        st.close()
        outs.append((out, base.cpu().numpy()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("storage", [fsb.STORAGE_F32, fsb.STORAGE_F16, fsb.STORAGE_BF16])
def test_laps_large_levels_match_cache(torch, ctx, storage):
    # levels wider than 512 take the streaming pyramid kernel in the laps and
    # fused modes;
    # odd, non-multiple-of-4 level sizes exercise its edge columns and rows.
    # FP32: laps and fused within one u8 step of cache on a handful of pixels;
    # reduced storage (they also keep their Laplacians in it): each mode within the
    # precision form's u8 bound of the oracle (1 for FP16, 2 for BF16)
    W, H, F = 1203, 917, 4
    frames, poses = synth_stack(torch, ctx, W, H, F, seed=21)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
    assert max(roi.width, roi.height) > 1024
    results = {}
    for mode in ("laps", "fused", "cache"):
        st = fsb.PyramidContrastStack(ctx, W, H, F, roi=roi, frames_per_batch=3, level_storage=storage,
                                      pass2_mode=mode)
        assert st.pass2_mode == mode
        for f, p in zip(frames, poses):
            st.add_frame(f, p)
        results[mode] = st.finish()
        st.close()
    if storage == fsb.STORAGE_F32:
        for m in ("laps", "fused"):
            assert close_outputs(results[m], results["cache"]), m
        return
    ref = oracle.stack_fuse(frames, [p.as_dict() for p in poses], roi.as_tuple(), jobs=8)
    bound = 1 if storage == fsb.STORAGE_F16 else 2
    for mode, out in results.items():
        assert np.abs(out.astype(np.int16) - ref.astype(np.int16)).max() <= bound, mode


def test_stack_errors(torch, ctx):
    W, H = 64, 48
    frames, poses = synth_stack(torch, ctx, W, H, 2, seed=2)
    with pytest.raises(fsb.FocusCudaError) as e:
        fsb.PyramidContrastStack(ctx, W, H, 2, contrast_window=4)
    assert e.value.code == "FS_ERR_INVALID"
    st = fsb.PyramidContrastStack(ctx, W, H, 2)
    st.add_frame(frames[0], poses[0])
    with pytest.raises(fsb.FocusCudaError) as e:
        st.finish()
    assert e.value.code == "FS_ERR_STATE"
    with pytest.raises(fsb.FocusCudaError) as e:
        st.add_frame(frames[1][:, :W // 2].copy(), poses[1])
    assert e.value.code == "FS_ERR_MISMATCH"
    st.add_frame(frames[1], poses[1])
    with pytest.raises(fsb.FocusCudaError) as e:
        st.add_frame(frames[1], poses[1])
    assert e.value.code == "FS_ERR_STATE"
    st.finish()
    with pytest.raises(fsb.FocusCudaError) as e:
        st.finish()
    assert e.value.code == "FS_ERR_STATE"
    st.close()
    with pytest.raises(fsb.FocusCudaError) as e:
        fsb.PyramidContrastStack(fsb.Context(0, hbm_budget_bytes=1024), 640, 480, 2)
    assert e.value.code == "FS_ERR_BUDGET"


def test_pipelined_finish_matches_sync(torch, ctx):
    # stack A's pass 2 is queued (finish_into_async) while stack B's frames
    # upload on the same context, every upload queued without a wait
    # (add_frame_async); both images equal the synchronous ones
    W, H, F = 640, 480, 5
    frames_a, poses_a = synth_stack(torch, ctx, W, H, F, seed=31)
    frames_b, poses_b = synth_stack(torch, ctx, W, H, F, seed=32)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses_a)
    roi_b = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses_b)

    def sync(frames, poses, r):
        st = fsb.PyramidContrastStack(ctx, W, H, F, roi=r)
        for f, p in zip(frames, poses):
            st.add_frame(f, p)
        out = st.finish()
        st.close()
        return out

    ref_a, ref_b = sync(frames_a, poses_a, roi), sync(frames_b, poses_b, roi_b)
    out_a = np.zeros_like(ref_a)
    out_b = np.zeros_like(ref_b)
    a = fsb.PyramidContrastStack(ctx, W, H, F, roi=roi)
    for f, p in zip(frames_a, poses_a):
        a.add_frame_async(f, p)
    a.finish_into_async(out_a)
    b = fsb.PyramidContrastStack(ctx, W, H, F, roi=roi_b)
    for f, p in zip(frames_b, poses_b):
        b.add_frame_async(f, p)
    a.wait()
    a.close()
    b.finish_into_async(out_b)
    b.close()  # waits for its own work
    assert np.array_equal(out_a, ref_a)
    assert np.array_equal(out_b, ref_b)


def test_stack_outliving_its_context(torch):
    # destroying a context releases its stacks' device memory; the stack
    # handles stay valid for fs_stack_destroy and report a state error
    c = fsb.Context(0)
    st = fsb.PyramidContrastStack(c, 64, 48, 2, aligned=True)
    c.close()
    with pytest.raises(fsb.FocusCudaError):
        st.add_frame(np.zeros((48, 64, 3), np.uint8))
    st.close()
