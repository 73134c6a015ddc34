"""fs_fuse_aligned_device_static, the fusion entry point that allocates
nothing, through the C ABI.

Some hosts cannot let a plugin allocate device memory while they run: a
server that reserved its HBM when it started and accounts for every byte, or
an interactive loop whose own kernels would stall behind the plugin's
cudaMalloc / cudaFree.  This entry point keeps every plane in a fixed
file-scope device array instead.  Checked here:
  * it gives the same bytes as the context-backed fuse-only path in the
    cache mode (the same kernels in the same order), on two calls
    in a row and with stacks of different sizes back to back, so planes one
    call leaves in the shared array never leak into the next;
  * it is within one u8 LSB of the oracle's fuse-only fusion;
  * it writes only the image columns of a padded output row;
  * device memory (free bytes and torch's allocator) does not change while it
    runs;
  * stacks beyond the array are rejected with a message.
This file is collected last so that a failure here comes after every other
test has run; it also passes when run alone in a fresh process.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

from __graft_entry__ import ROOT, load_package

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

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


class StaticCall:
    """Device inputs and output of one static fusion, allocated up front so
    that the call itself is the only thing that runs."""

    def __init__(self, torch, frames, window, pad=0):
        h, w, c = frames[0].shape
        self.torch, self.w, self.h, self.c, self.window = torch, w, h, c, window
        self.dev = [torch.from_numpy(f).to("cuda:0") for f in frames]
        self.stride = w * 3 + pad
        self.out = torch.full((h, self.stride), 7, dtype=torch.uint8, device="cuda:0")
        self.ptrs = (ctypes.c_void_p * len(self.dev))(*[t.data_ptr() for t in self.dev])
        self.strides = (ctypes.c_size_t * len(self.dev))(*[w * c] * len(self.dev))
        self.err = ctypes.create_string_buffer(512)

    def run(self):
        stream = self.torch.cuda.current_stream().cuda_stream
        rc = fsb._lib.lib().fs_fuse_aligned_device_static(
            self.ptrs, self.strides, len(self.dev), self.w, self.h, self.c, self.window, self.out.data_ptr(),
            self.stride, stream, self.err, len(self.err))
        assert rc == 0, self.err.value.decode()

    def result(self):
        self.torch.cuda.synchronize()
        rows = self.out.cpu().numpy()
        return rows[:, :self.w * 3].reshape(self.h, self.w, 3).copy(), rows[:, self.w * 3:].copy()


def context_fuse(ctx, frames, window):
    """The context-backed fuse-only path in the cache mode, which runs the
    kernels of the static path in the same order."""
    h, w, c = frames[0].shape
    with fsb.PyramidContrastStack(ctx, w, h, len(frames), channels=c, contrast_window=window, aligned=True,
                                  pass2_mode="cache") as st:
        for im in frames:
            st.add_frame(im)
        return st.finish()


def static_fuse(torch, frames, window):
    call = StaticCall(torch, frames, window)
    call.run()
    return call.result()[0]


CASES = [
    # (seed, width, height, frames, channels, window)
    (11, 320, 240, 4, 4, 5),
    (12, 512, 512, 8, 3, 7),   # the largest stack the 40 MiB scratch takes
    (13, 97, 61, 3, 4, 3),
]


def test_static_fusion_equals_context_path_back_to_back(torch, ctx):
    for seed, w, h, n, c, win in CASES + CASES[:1]:
        frames = aligned_stack(seed, w, h, n, c)
        got = static_fuse(torch, frames, win)
        want = context_fuse(ctx, frames, win)
        diff = np.abs(got.astype(np.int16) - want.astype(np.int16))
        assert np.array_equal(got, want), ((w, h, n, c), int(diff.max()), int((diff > 0).sum()))
    # two calls in a row on the same stack give the same bytes
    frames = aligned_stack(CASES[0][0], *CASES[0][1:5])
    a = static_fuse(torch, frames, CASES[0][5])
    b = static_fuse(torch, frames, CASES[0][5])
    assert np.array_equal(a, b)


@pytest.mark.parametrize("case", [CASES[0], CASES[2]])
def test_static_fusion_within_one_lsb_of_the_oracle(torch, case):
    seed, w, h, n, c, win = case
    frames = aligned_stack(seed, w, h, n, c)
    got = static_fuse(torch, frames, win)
    _, base = oracle.fuse_aligned(frames, window=win, want_base=True)
    ref8 = np.clip(np.floor(base + 0.5), 0, 255)
    assert np.abs(got.astype(np.int32) - ref8.astype(np.int32)).max() <= 1


def test_static_fusion_padded_output_rows(torch, ctx):
    seed, w, h, n, c, win = CASES[0]
    frames = aligned_stack(seed, w, h, n, c)
    call = StaticCall(torch, frames, win, pad=64)
    call.run()
    img, pad = call.result()
    assert np.array_equal(img, context_fuse(ctx, frames, win))
    assert (pad == 7).all(), "bytes past the image columns were written"


def test_static_fusion_allocates_no_device_memory(torch):
    calls = [StaticCall(torch, aligned_stack(seed, w, h, n, c), win) for seed, w, h, n, c, win in CASES]
    calls[0].run()  # the first call on the device loads the module and its 40 MiB array
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    reserved0, allocated0 = torch.cuda.memory_reserved(0), torch.cuda.memory_allocated(0)
    for _ in range(2):
        for call in calls:
            call.run()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"device free memory moved by {free0 - free1} bytes"
    assert torch.cuda.memory_reserved(0) == reserved0
    assert torch.cuda.memory_allocated(0) == allocated0


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
