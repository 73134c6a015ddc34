"""fs_fuse_aligned_device_static (static-scratch fusion, no allocation)
against the context-backed fuse-only path (fs_fuse_stack through
fuse_aligned_images), through the C ABI.

Both run the same kernels in the same order, so the outputs are expected to
be identical; the bar is the suite's u8 tolerance (1 LSB).  Calls are made
back to back on one stream, with stacks of different sizes, so planes left
in the shared scratch by one call must not leak into the next.
"""
import ctypes

import numpy as np
import pytest

from __graft_entry__ import load_package

fsb = load_package()
pytestmark = pytest.mark.gpu

FS_ERR_UNSUPPORTED = 8


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


def aligned_stack(seed, w, h, count, channels):
    """Frames with smooth structure, local detail that differs per frame and,
    for RGBA, transparent borders of different widths (partial support)."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    frames = []
    for k in range(count):
        base = 128 + 60 * np.sin(xx / (9 + k) + k) * np.cos(yy / (13 + 2 * k))
        detail = rng.normal(0, 6 + 10 * (k % 3), (h, w)).astype(np.float32)
        rgb = np.stack([base + detail, base * 0.8 + detail, 255 - base + detail], axis=-1)
        img = np.clip(np.rint(rgb), 0, 255).astype(np.uint8)
        if channels == 4:
            alpha = np.full((h, w, 1), 255, np.uint8)
            m = 3 + 4 * k
            alpha[:m] = 0
            alpha[:, w - m:] = 0
            img = np.concatenate([img, alpha], axis=-1)
        frames.append(np.ascontiguousarray(img))
    return frames


def static_fuse(torch, frames, window):
    h, w, c = frames[0].shape
    dev = [torch.from_numpy(f).to("cuda:0") for f in frames]
    out = torch.full((h, w, 3), 7, dtype=torch.uint8, device="cuda:0")
    ptrs = (ctypes.c_void_p * len(dev))(*[t.data_ptr() for t in dev])
    strides = (ctypes.c_size_t * len(dev))(*[w * c] * len(dev))
    err = ctypes.create_string_buffer(512)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fsb._lib.lib().fs_fuse_aligned_device_static(ptrs, strides, len(dev), w, h, c, window, out.data_ptr(),
                                                      w * 3, stream, err, len(err))
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def context_fuse(ctx, frames, window):
    return fsb.fuse_aligned_images(ctx, frames, contrast_window=window)


CASES = [
    # (seed, width, height, frames, channels, window)
    (11, 320, 240, 4, 4, 5),
    (12, 512, 512, 8, 3, 7),   # the largest stack the 40 MiB scratch takes
    (13, 97, 61, 3, 4, 3),
]


def test_static_fusion_matches_context_path_back_to_back(torch, ctx):
    results = []
    for seed, w, h, n, c, win in CASES + CASES[:1]:
        frames = aligned_stack(seed, w, h, n, c)
        got = static_fuse(torch, frames, win)
        want = context_fuse(ctx, frames, win)
        diff = np.abs(got.astype(np.int16) - want.astype(np.int16))
        results.append((w, h, n, c, int(diff.max()), int((diff > 0).sum())))
        assert diff.max() <= 1, results
    # two calls in a row on the same stack give the same bytes
    frames = aligned_stack(CASES[0][0], *CASES[0][1:5])
    a = static_fuse(torch, frames, CASES[0][5])
    b = static_fuse(torch, frames, CASES[0][5])
    assert np.array_equal(a, b)


def test_static_fusion_rejects_stacks_beyond_scratch(torch):
    lib = fsb._lib.lib()
    dummy = torch.zeros(16, dtype=torch.uint8, device="cuda:0")
    err = ctypes.create_string_buffer(512)
    for n, w, h in ((8, 700, 700), (9, 64, 64), (2, 9000, 16)):
        ptrs = (ctypes.c_void_p * n)(*[dummy.data_ptr()] * n)
        strides = (ctypes.c_size_t * n)(*[w * 3] * n)
        rc = lib.fs_fuse_aligned_device_static(ptrs, strides, n, w, h, 3, 5, dummy.data_ptr(), w * 3, None, err,
                                               len(err))
        assert rc == FS_ERR_UNSUPPORTED, (n, w, h, rc)
        assert err.value, "no message"
