"""JPEG frames decoded on the device, against PIL's libjpeg (the decoder the
reference links, src/image_io.zig:160-173; PIL's decode of the reference's
fixture 0001.jpg equals the reference's identity-remap golden byte for byte).

Bar: byte-identical RGB for baseline files at 4:4:4, 4:2:2 and 4:2:0, with
and without restart markers, at sizes that are not multiples of the MCU; a
stack fed JPEG frames gives exactly the bytes of the same stack fed the
decoded frames.
"""
import io

import numpy as np
import pytest

from __graft_entry__ import load_package

fsb = load_package()

PIL = pytest.importorskip("PIL.Image")


def encode(img, quality=90, subsampling=2, restart_rows=0, progressive=False):
    b = io.BytesIO()
    kw = dict(format="JPEG", quality=quality, subsampling=subsampling, progressive=progressive)
    if restart_rows:
        kw["restart_marker_rows"] = restart_rows
    PIL.fromarray(img).save(b, **kw)
    return b.getvalue()


def pil_decode(data):
    return np.asarray(PIL.open(io.BytesIO(data)).convert("RGB"))


def test_info_and_unsupported_files():
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, (37, 53, 3), dtype=np.uint8)
    assert fsb.jpeg_info(encode(img)) == (53, 37)
    with pytest.raises(fsb.FocusCudaError) as e:
        fsb.jpeg_info(encode(img, progressive=True))
    assert e.value.code == "FS_ERR_UNSUPPORTED"
    with pytest.raises(fsb.FocusCudaError):
        fsb.jpeg_info(b"not a jpeg")


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


def scene(torch, ctx, w, h, seed, k=0):
    buf = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda:0")
    pose = fsb.synth_frame_device(ctx, seed, fsb.SCENE_SMALL, w, h, k, 4, buf, w * 3)
    return buf.cpu().numpy(), pose


@pytest.mark.gpu
@pytest.mark.parametrize("subsampling", [0, 1, 2])
@pytest.mark.parametrize("restart_rows", [0, 1, 3])
@pytest.mark.parametrize("w,h", [(333, 219), (64, 48), (17, 9)])
def test_decode_matches_libjpeg(torch, ctx, subsampling, restart_rows, w, h):
    img, _ = scene(torch, ctx, w, h, seed=w + subsampling)
    data = encode(img, quality=88, subsampling=subsampling, restart_rows=restart_rows)
    got = fsb.decode_jpeg(ctx, data)
    want = pil_decode(data)
    assert np.array_equal(got, want), int((got != want).any(-1).sum())


@pytest.mark.gpu
def test_decode_noise_and_extremes(torch, ctx):
    rng = np.random.default_rng(5)
    img = rng.integers(0, 256, (120, 200, 3), dtype=np.uint8)
    img[:40] = 0
    img[40:60] = 255
    for q in (50, 95, 100):
        data = encode(img, quality=q, subsampling=2, restart_rows=2)
        assert np.array_equal(fsb.decode_jpeg(ctx, data), pil_decode(data)), q


@pytest.mark.gpu
def test_stack_fed_jpeg_frames_equals_decoded_frames(torch, ctx):
    W, H, F = 640, 480, 4
    frames, poses, files = [], [], []
    for k in range(F):
        img, pose = scene(torch, ctx, W, H, seed=3, k=k)
        data = encode(img, quality=92, subsampling=2, restart_rows=1)
        files.append(data)
        frames.append(pil_decode(data))
        poses.append(pose)
    roi = fsb.compute_common_overlap_roi([True] * F, [W] * F, [H] * F, poses)
    want = fsb.fuse_remapped_images(ctx, frames, poses, roi)
    st = fsb.PyramidContrastStack(ctx, W, H, F, roi=roi)
    for data, pose in zip(files, poses):
        st.add_frame_jpeg(data, pose)
    got = st.finish()
    st.close()
    assert np.array_equal(got, want)
