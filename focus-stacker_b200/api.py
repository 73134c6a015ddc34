"""Host-side mirror of the reference's operator interface for the remap +
pyramid-contrast fusion path, over libfocuscuda.so.

Names and argument meanings follow the reference (asingleoat/focus-stacker):
  * ImagePose / Rect                 src/optimize.zig:32-48, src/remap.zig:573-578
  * compute_common_overlap_roi       src/remap.zig:585-633 (None = no overlap)
  * remap_rigid_image                src/remap.zig:166-204 (RGB/gray u8 -> +alpha)
  * Method / parse_method            src/fuse/config.zig:10-24, 281-287, plus
                                     the drop-in "cuda-pyramid-contrast"
  * fuse_remapped_images             stack path, src/stack/pipeline.zig:314-605
  * fuse_aligned_images              fuse-only path, src/fuse/pipeline.zig:148-445
Errors are raised as FocusCudaError carrying the C status (the reference's
Zig error unions map onto the same categories: InvalidValue, OutOfMemory,
MismatchedImageSizes, ...).  Host arrays are numpy; device buffers are any
object with data_ptr() (e.g. a torch CUDA tensor) or a raw integer pointer.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass, fields
from typing import List, Optional, Sequence

import numpy as np

from . import _lib

L = _lib.lib


class FocusCudaError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = status
        self.code = _lib.STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.code}: {message}" if message else self.code)


@dataclass
class ImagePose:
    yaw: float = 0.0
    pitch: float = 0.0
    roll: float = 0.0
    hfov_delta: float = 0.0
    trans_x: float = 0.0
    trans_y: float = 0.0
    trans_z: float = 0.0
    translation_plane_yaw: float = 0.0
    translation_plane_pitch: float = 0.0
    radial_a: float = 0.0
    radial_b: float = 0.0
    radial_c: float = 0.0
    center_shift_x: float = 0.0
    center_shift_y: float = 0.0
    base_hfov_degrees: float = 50.0

    def to_c(self) -> _lib.FsPose:
        return _lib.FsPose(*[float(getattr(self, f.name)) for f in fields(self)])

    @staticmethod
    def from_c(p: _lib.FsPose) -> "ImagePose":
        return ImagePose(*[getattr(p, f.name) for f in fields(ImagePose)])

    def as_dict(self) -> dict:
        return {f.name: float(getattr(self, f.name)) for f in fields(self)}


@dataclass(frozen=True)
class Rect:
    left: int
    top: int
    right: int
    bottom: int

    @property
    def width(self) -> int:
        return self.right - self.left

    @property
    def height(self) -> int:
        return self.bottom - self.top

    def to_c(self) -> _lib.FsRect:
        return _lib.FsRect(self.left, self.top, self.right, self.bottom)

    def as_tuple(self):
        return (self.left, self.top, self.right, self.bottom)


def _pose(p) -> ImagePose:
    if p is None:
        return ImagePose()
    if isinstance(p, ImagePose):
        return p
    if isinstance(p, dict):
        return ImagePose(**p)
    return ImagePose(**{f.name: getattr(p, f.name) for f in fields(ImagePose)})


class Method(enum.Enum):
    """Fusion methods of the reference CLIs plus the CUDA drop-in."""
    HARDMASK_CONTRAST = "hardmask-contrast"
    SOFTMASK_CONTRAST = "softmask-contrast"
    PYRAMID_CONTRAST = "pyramid-contrast"
    HYBRID_PYRAMID_CONTRAST = "hybrid-pyramid-contrast"
    CUDA_PYRAMID_CONTRAST = "cuda-pyramid-contrast"
    CUDA_HYBRID_PYRAMID_CONTRAST = "cuda-hybrid-pyramid-contrast"

    def cli_name(self) -> str:
        return self.value


def parse_method(value: str) -> Method:
    """src/fuse/config.zig:281-287; unknown names raise ValueError (InvalidValue)."""
    for m in Method:
        if m.value == value:
            return m
    raise ValueError("InvalidValue")


def parse_window_size(value: str) -> int:
    """src/fuse/config.zig:295-299: odd and >= 3."""
    try:
        v = int(value, 10)
    except ValueError:
        raise ValueError("InvalidValue") from None
    if v <= 0 or v < 3 or (v & 1) == 0:
        raise ValueError("InvalidValue")
    return v


def _check(rc: int, ctx_handle=None):
    if rc != _lib.FS_OK:
        msg = ""
        if ctx_handle:
            raw = L().fs_last_error(ctx_handle)
            msg = raw.decode() if raw else ""
        raise FocusCudaError(rc, msg)


def _ptr(buf) -> int:
    if isinstance(buf, int):
        return buf
    if hasattr(buf, "data_ptr"):
        return int(buf.data_ptr())
    raise TypeError("expected a device buffer with data_ptr() or an integer pointer")


class Context:
    """One CUDA device context (fs_ctx): stream, HBM budget, kernel accounting."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        h = ctypes.c_void_p()
        rc = L().fs_create(device, hbm_budget_bytes, ctypes.byref(h))
        if rc != _lib.FS_OK:
            raise FocusCudaError(rc, "fs_create")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            L().fs_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self) -> str:
        raw = L().fs_last_error(self.handle)
        return raw.decode() if raw else ""

    def synchronize(self):
        _check(L().fs_ctx_synchronize(self.handle), self.handle)

    def device_bytes(self) -> int:
        return int(L().fs_ctx_device_bytes(self.handle))

    def budget(self) -> int:
        """The context's HBM budget in bytes."""
        return int(L().fs_ctx_budget(self.handle))

    def trim(self):
        _check(L().fs_ctx_trim(self.handle), self.handle)

    def reserve(self, nbytes: int):
        """Grow the device's shared memory pool by nbytes (kept cached)."""
        _check(L().fs_ctx_reserve(self.handle, int(nbytes)), self.handle)

    def set_budget(self, hbm_budget_bytes: int):
        """Change the HBM budget later allocations and pass-2 mode choices use."""
        _check(L().fs_ctx_set_budget(self.handle, int(hbm_budget_bytes)), self.handle)

    def set_level_schedule(self, fuse_min_tiles: int = 0, tail_side: int = 0):
        """Level schedule of the split-pyramid stacks begun from now on: levels
        of at least fuse_min_tiles 64x32 tiles blend and REDUCE their masks in
        one pass (0: the default 1184), levels with both sides at most
        tail_side (0: 64) run as the small-level tail.  Same bytes either way."""
        _check(L().fs_ctx_set_level_schedule(self.handle, int(fuse_min_tiles), int(tail_side)), self.handle)

    def stream_handle(self) -> int:
        """cudaStream_t of the context (e.g. for torch.cuda.ExternalStream)."""
        v = ctypes.c_void_p()
        _check(L().fs_ctx_stream(self.handle, ctypes.byref(v)), self.handle)
        return int(v.value or 0)

    def launch_count(self) -> int:
        return int(L().fs_ctx_launch_count(self.handle))

    def set_kernel_timing(self, enable: bool):
        _check(L().fs_ctx_set_kernel_timing(self.handle, 1 if enable else 0), self.handle)

    def kernel_stats(self, kernel: str):
        n = ctypes.c_uint64()
        ms = ctypes.c_double()
        _check(L().fs_ctx_kernel_stats(self.handle, kernel.encode(), ctypes.byref(n), ctypes.byref(ms)), self.handle)
        return int(n.value), float(ms.value)


# ------------------------------------------------------------ pose utilities
def compute_common_overlap_roi(remap_active: Sequence[bool], widths: Sequence[int], heights: Sequence[int],
                               poses: Sequence) -> Optional[Rect]:
    n = len(poses)
    parr = (_lib.FsPose * max(1, n))(*[_pose(p).to_c() for p in poses])
    w = (ctypes.c_uint32 * max(1, n))(*widths)
    h = (ctypes.c_uint32 * max(1, n))(*heights)
    a = (ctypes.c_uint8 * max(1, n))(*[1 if x else 0 for x in remap_active])
    out = _lib.FsRect()
    has = ctypes.c_int()
    _check(L().fs_compute_roi(parr, w, h, a, n, ctypes.byref(out), ctypes.byref(has)))
    return Rect(out.left, out.top, out.right, out.bottom) if has.value else None


def inverse_map_points(pose, width: int, height: int, xy: np.ndarray) -> np.ndarray:
    xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1, 2)
    out = np.zeros_like(xy)
    p = _pose(pose).to_c()
    _check(L().fs_inverse_map_points(ctypes.byref(p), width, height, xy.shape[0],
                                     xy.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return out


def forward_map_points(pose, width: int, height: int, xy: np.ndarray) -> np.ndarray:
    """Source-frame points -> aligned-frame points (the reference's transformPoint)."""
    xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1, 2)
    out = np.zeros_like(xy)
    p = _pose(pose).to_c()
    _check(L().fs_forward_map_points(ctypes.byref(p), width, height, xy.shape[0],
                                     xy.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return out


def exact_expand_divisor(x: int, y: int, src_w: int, src_h: int) -> float:
    return float(L().fs_exact_expand_divisor(x, y, src_w, src_h))


# ---------------------------------------------------------------------- remap
def remap_rigid_image(ctx: Context, src: np.ndarray, pose, roi: Optional[Rect] = None) -> np.ndarray:
    """src: HxW (gray) or HxWx3, uint8 or uint16 (remapU8 / remapU16).
    Returns the ROI-sized image with an extra alpha channel, same sample type."""
    src = np.ascontiguousarray(src)
    if src.dtype not in (np.uint8, np.uint16):
        raise FocusCudaError(8, "samples must be uint8 or uint16")
    h, w = src.shape[:2]
    ch = 1 if src.ndim == 2 else src.shape[2]
    r = roi or Rect(0, 0, w, h)
    out = np.zeros((r.height, r.width, ch + 1), src.dtype)
    p = _pose(pose).to_c()
    fn = L().fs_remap_frame16 if src.dtype == np.uint16 else L().fs_remap_frame
    rc = fn(ctx.handle, src.ctypes.data, src.strides[0], w, h, ch, ctypes.byref(p), ctypes.byref(r.to_c()),
            out.ctypes.data, out.strides[0])
    _check(rc, ctx.handle)
    return out


def remap_rigid_image_device(ctx: Context, src, src_stride: int, width: int, height: int, channels: int, pose,
                             roi: Optional[Rect], dst, dst_stride: int):
    p = _pose(pose).to_c()
    r = roi.to_c() if roi else None
    rc = L().fs_remap_frame_device(ctx.handle, _ptr(src), src_stride, width, height, channels, ctypes.byref(p),
                                   ctypes.byref(r) if r else None, _ptr(dst), dst_stride)
    _check(rc, ctx.handle)


# ----------------------------------------------------------------------- JPEG
def jpeg_info(data: bytes):
    """(width, height) of a JPEG file the device decoder takes; raises
    FocusCudaError(FS_ERR_UNSUPPORTED) for other files."""
    w, h = ctypes.c_uint32(), ctypes.c_uint32()
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    _check(L().fs_jpeg_info(buf, len(data), ctypes.byref(w), ctypes.byref(h)))
    return w.value, h.value


def decode_jpeg(ctx: Context, data: bytes) -> np.ndarray:
    """Decode a JPEG file on the device (libjpeg's default output: islow IDCT,
    fancy upsampling); returns HxWx3 uint8."""
    w, h = jpeg_info(data)
    out = np.zeros((h, w, 3), np.uint8)
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    _check(L().fs_decode_jpeg(ctx.handle, buf, len(data), out.ctypes.data, out.strides[0], 0), ctx.handle)
    return out


def decode_jpeg_device(ctx: Context, data: bytes, dst, dst_stride: int):
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    _check(L().fs_decode_jpeg(ctx.handle, buf, len(data), _ptr(dst), dst_stride, 1), ctx.handle)


# --------------------------------------------------------------------- fusion
PASS2_MODES = ("cache", "resident", "refetch", "laps", "fused")
# fs_stack_set_method: the fusion methods the stack runs on the device, and
# the default weight of the hard image's levels (--hybrid-sharpness,
# src/fuse/pyramid.zig:11)
FUSION_METHODS = ("pyramid-contrast", "hybrid-pyramid-contrast")
HYBRID_SHARPNESS = 0.35
BUFFER_WEIGHT_SUM, BUFFER_UNION, BUFFER_ACCUMULATOR, BUFFER_HARD = 0, 1, 2, 3


class DeviceBuffer:
    """A device buffer of a stack, exposed through __cuda_array_interface__
    (torch.as_tensor(buf, device="cuda") is a view, not a copy); `width` and
    `height` give the valid region inside the pitched rows.  Keeps its stack
    alive."""

    def __init__(self, ptr: int, shape, typestr: str, width: int, height: int, owner):
        self.ptr, self.shape, self.typestr = ptr, tuple(shape), typestr
        self.width, self.height, self._owner = width, height, owner

    @property
    def __cuda_array_interface__(self):
        return {"shape": self.shape, "typestr": self.typestr, "data": (self.ptr, False), "version": 2,
                "strides": None}


def stack_desc(src_width: int, src_height: int, frame_count: int, roi: Optional[Rect] = None, channels: int = 3,
               contrast_window: int = 5, aligned: bool = False, frames_per_batch: int = 0,
               level_storage: int = 0, sample_bits: int = 8) -> _lib.FsStackDesc:
    d = _lib.FsStackDesc()
    d.src_width, d.src_height = src_width, src_height
    d.has_roi = 1 if roi is not None else 0
    if roi is not None:
        d.roi = roi.to_c()
    d.channels = channels
    d.sample_bits = sample_bits
    d.frame_count = frame_count
    d.contrast_window = contrast_window
    d.input_is_aligned = 1 if aligned else 0
    d.level_storage = level_storage
    d.frames_per_batch = frames_per_batch
    return d


def stack_mode_bytes(desc: _lib.FsStackDesc, mode: str, host_frames: bool = True) -> int:
    """Device bytes of a stack in pass-2 mode `mode`; allocates nothing."""
    b = ctypes.c_uint64()
    _check(L().fs_stack_mode_bytes(ctypes.byref(desc), PASS2_MODES.index(mode), 1 if host_frames else 0,
                                   ctypes.byref(b)))
    return int(b.value)


def stack_footprint(desc: _lib.FsStackDesc, available_bytes: int, host_frames: bool = True):
    """(device bytes, pass-2 mode, fits) of a stack when `available_bytes` of
    budget are free; allocates nothing."""
    b, m = ctypes.c_uint64(), ctypes.c_int32()
    rc = L().fs_stack_footprint(ctypes.byref(desc), int(available_bytes), 1 if host_frames else 0, ctypes.byref(b),
                                ctypes.byref(m))
    if rc not in (_lib.FS_OK, 3):
        raise FocusCudaError(rc, "fs_stack_footprint")
    return int(b.value), PASS2_MODES[m.value], rc == _lib.FS_OK


class PyramidContrastStack:
    """Streaming two-pass pyramid-contrast fusion on the device (fs_stack).

    add_frame / add_frame_device run pass 1 as frames arrive (in the
    reference's active-frame order); finish runs pass 2 and the collapse."""

    def __init__(self, ctx: Context, src_width: int, src_height: int, frame_count: int, roi: Optional[Rect] = None,
                 channels: int = 3, contrast_window: int = 5, aligned: bool = False, frames_per_batch: int = 0,
                 level_storage: int = 0, pass2_mode: Optional[str] = None, sample_bits: int = 8,
                 method: str = "pyramid-contrast", hybrid_sharpness: float = HYBRID_SHARPNESS):
        """pass2_mode: None picks the mode from the context's budget; "cache",
        "resident", "refetch", "laps" or "fused" imposes one.  sample_bits 16: uint16
        frames in and a uint16 image out (FP32 levels; resident / refetch)."""
        self.ctx = ctx
        d = stack_desc(src_width, src_height, frame_count, roi, channels, contrast_window, aligned, frames_per_batch,
                       level_storage, sample_bits)
        self.dtype = np.uint16 if sample_bits == 16 else np.uint8
        self.desc = d
        h = ctypes.c_void_p()
        mode = -1 if pass2_mode is None else PASS2_MODES.index(pass2_mode)
        _check(L().fs_stack_begin_mode(ctx.handle, ctypes.byref(d), mode, ctypes.byref(h)), ctx.handle)
        self.handle = h
        if method not in FUSION_METHODS:
            self.close()
            raise FocusCudaError(1, f"unknown fusion method {method!r}")
        if method != "pyramid-contrast":
            _check(L().fs_stack_set_method(h, FUSION_METHODS.index(method), hybrid_sharpness), ctx.handle)
        w, hh = ctypes.c_uint32(), ctypes.c_uint32()
        L().fs_stack_output_size(h, ctypes.byref(w), ctypes.byref(hh))
        self.out_width, self.out_height = w.value, hh.value
        self._keep = []

    PASS2_MODES = PASS2_MODES

    @property
    def pass2_mode(self) -> str:
        """Where pass 2 takes its frames from (chosen from the HBM budget)."""
        return self.PASS2_MODES[L().fs_stack_pass2_mode(self.handle)]

    def set_base_output(self, dst, row_stride_elems: int):
        """Also write the collapsed FP32 base (RGB, device buffer) during finish."""
        self._keep.append(dst)
        _check(L().fs_stack_set_base_output(self.handle, _ptr(dst), row_stride_elems), self.ctx.handle)

    def add_frame(self, pixels: np.ndarray, pose=None):
        pixels = np.ascontiguousarray(pixels)
        if pixels.dtype != self.dtype:
            raise FocusCudaError(7, "MismatchedImageFormats")
        p = _pose(pose).to_c() if pose is not None else None
        rc = L().fs_stack_add_frame(self.handle, pixels.ctypes.data, pixels.strides[0],
                                    ctypes.byref(p) if p is not None else None)
        _check(rc, self.ctx.handle)

    def add_frame_async(self, pixels: np.ndarray, pose=None):
        """add_frame without waiting for the upload; `pixels` (best pinned
        memory) is kept referenced and must not change until finish or wait
        has returned."""
        pixels = np.ascontiguousarray(pixels)
        if pixels.dtype != self.dtype:
            raise FocusCudaError(7, "MismatchedImageFormats")
        self._keep.append(pixels)
        p = _pose(pose).to_c() if pose is not None else None
        rc = L().fs_stack_add_frame_async(self.handle, pixels.ctypes.data, pixels.strides[0],
                                          ctypes.byref(p) if p is not None else None)
        _check(rc, self.ctx.handle)

    def add_frame_jpeg(self, data: bytes, pose=None):
        """A frame given as a JPEG file, decoded on the device
        (fs_stack_add_frame_jpeg)."""
        p = _pose(pose).to_c() if pose is not None else None
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        rc = L().fs_stack_add_frame_jpeg(self.handle, buf, len(data), ctypes.byref(p) if p is not None else None)
        _check(rc, self.ctx.handle)

    def add_frame_device(self, buf, row_stride: int, pose=None):
        p = _pose(pose).to_c() if pose is not None else None
        self._keep.append(buf)
        rc = L().fs_stack_add_frame_device(self.handle, _ptr(buf), row_stride, ctypes.byref(p) if p is not None else None)
        _check(rc, self.ctx.handle)

    def finish(self, refetch=None) -> np.ndarray:
        out = np.zeros((self.out_height, self.out_width, 3), self.dtype)
        self.finish_into(out, refetch)
        return out

    def finish_into(self, out: np.ndarray, refetch=None):
        cb = self._make_cb(refetch)
        rc = L().fs_stack_finish(self.handle, cb, None, out.ctypes.data, out.strides[0])
        _check(rc, self.ctx.handle)

    def finish_device(self, dst, dst_stride: int, refetch=None):
        cb = self._make_cb(refetch)
        _check(L().fs_stack_finish_device(self.handle, cb, None, _ptr(dst), dst_stride), self.ctx.handle)

    def finish_into_async(self, out: np.ndarray, refetch=None):
        """Queue pass 2, the collapse and the copy of the fused image into
        `out` (best pinned host memory) and return; `wait()` blocks until the
        image is there.  The next stack on the same context can be fed in the
        meantime, so that its uploads overlap this stack's pass 2."""
        cb = self._make_cb(refetch)
        self._keep.append(out)
        rc = L().fs_stack_finish_async(self.handle, cb, None, out.ctypes.data, out.strides[0])
        _check(rc, self.ctx.handle)

    def wait(self):
        _check(L().fs_stack_wait(self.handle), self.ctx.handle)

    # ---------------------------------------------- phases (frame shards)
    def set_frame_total(self, frame_total: int):
        """Frames of the whole stack when this one holds a shard of them."""
        _check(L().fs_stack_set_frame_total(self.handle, frame_total), self.ctx.handle)

    def end_pass1(self):
        _check(L().fs_stack_end_pass1(self.handle), self.ctx.handle)

    def blend(self, refetch=None):
        cb = self._make_cb(refetch)
        _check(L().fs_stack_blend(self.handle, cb, None), self.ctx.handle)

    def collapse(self) -> np.ndarray:
        out = np.zeros((self.out_height, self.out_width, 3), self.dtype)
        _check(L().fs_stack_collapse(self.handle, out.ctypes.data_as(ctypes.c_void_p), out.strides[0], 0),
               self.ctx.handle)
        return out

    def collapse_device(self, dst, dst_stride: int):
        _check(L().fs_stack_collapse(self.handle, _ptr(dst), dst_stride, 1), self.ctx.handle)

    def buffer(self, which: int, level: int = 0) -> "DeviceBuffer":
        """Device view (with __cuda_array_interface__) of the weight sum, the
        union support or a level's accumulator (3 x height x pitch)."""
        p, b = ctypes.c_void_p(), ctypes.c_uint64()
        pitch, w, h = ctypes.c_int64(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(L().fs_stack_buffer(self.handle, which, level, ctypes.byref(p), ctypes.byref(b), ctypes.byref(pitch),
                                   ctypes.byref(w), ctypes.byref(h)), self.ctx.handle)
        if which == BUFFER_ACCUMULATOR:
            shape, typestr = (3, h.value, pitch.value), "<f4"
        elif which == BUFFER_WEIGHT_SUM:
            shape, typestr = (h.value, pitch.value), "<f4"
        elif which == BUFFER_HARD:
            shape, typestr = (h.value, pitch.value), "<i4"  # RGBA words (bit pattern of u32)
        else:
            shape, typestr = (h.value, pitch.value), "|u1"
        return DeviceBuffer(int(p.value), shape, typestr, w.value, h.value, self)

    def _make_cb(self, refetch):
        held = []

        def cb(user, index, pixels, stride):
            try:
                arr = np.ascontiguousarray(refetch(int(index)))
                held.append(arr)
                pixels[0] = arr.ctypes.data
                stride[0] = arr.strides[0]
                return 0
            except Exception:
                return 1

        self._cb_hold = (_lib.FETCH_CB(cb) if refetch else _lib.FETCH_CB(0), held)
        return self._cb_hold[0]

    def close(self):
        if self.handle:
            L().fs_stack_destroy(self.handle)
            self.handle = None
            self._keep = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fuse_remapped_images(ctx: Context, sources: Sequence[np.ndarray], poses: Sequence, roi: Optional[Rect],
                         contrast_window: int = 5, frames_per_batch: int = 0, method: str = "pyramid-contrast",
                         hybrid_sharpness: float = HYBRID_SHARPNESS) -> np.ndarray:
    """Stack path: remap every active frame through its pose into the ROI and
    fuse with pyramid-contrast (runCollapsedPyramidStackPass), or with
    method="hybrid-pyramid-contrast" the hybrid branch of the same driver."""
    h, w = sources[0].shape[:2]
    bits = 16 if sources[0].dtype == np.uint16 else 8
    with PyramidContrastStack(ctx, w, h, len(sources), roi=roi, channels=3, contrast_window=contrast_window,
                              frames_per_batch=frames_per_batch, sample_bits=bits, method=method,
                              hybrid_sharpness=hybrid_sharpness) as st:
        for src, pose in zip(sources, poses):
            if src.shape[:2] != (h, w):
                raise FocusCudaError(7, "MismatchedImageSizes")
            st.add_frame(src, pose)
        return st.finish()


def fuse_aligned_images(ctx: Context, images: Sequence[np.ndarray], contrast_window: int = 5,
                        frames_per_batch: int = 0) -> np.ndarray:
    """Fuse-only path (focus_fuse_zig): pre-aligned RGB or RGBA frames."""
    h, w, c = images[0].shape
    bits = 16 if images[0].dtype == np.uint16 else 8
    with PyramidContrastStack(ctx, w, h, len(images), channels=c, contrast_window=contrast_window, aligned=True,
                              frames_per_batch=frames_per_batch, sample_bits=bits) as st:
        for im in images:
            if im.shape != (h, w, c):
                raise FocusCudaError(7, "MismatchedImageSizes" if im.shape[:2] != (h, w) else "MismatchedImageFormats")
            st.add_frame(im)
        return st.finish()


# ------------------------------------------------------------- batched form
@dataclass
class BatchStack:
    """One stack of a StackBatch: device frames (objects with data_ptr(), all
    of one size), their poses (None for aligned input), the ROI (None: full
    frame) and a device output of ROI size (RGB u8)."""
    frames: Sequence
    poses: Optional[Sequence]
    roi: Optional[Rect]
    out: object
    width: int
    height: int
    channels: int = 3
    aligned: bool = False


class StackBatch:
    """Batched form (fs_batch_*): many independent stacks over device frames,
    spread over `lanes` streams and run as one captured CUDA graph from the
    second run on.  Frames are read at the same addresses on every run."""

    def __init__(self, ctx: Context, stacks: Sequence[BatchStack], lanes: int = 4, pass2_mode: int = -1,
                 contrast_window: int = 5, frames_per_batch: int = 0, level_storage: int = 0,
                 fuse_min_tiles: int = 0, tail_side: int = 0):
        self.ctx = ctx
        # the lanes' stacks take the context's level schedule at creation
        ctx.set_level_schedule(fuse_min_tiles, tail_side)
        n = len(stacks)
        descs = (_lib.FsStackDesc * n)()
        frame_lists, pose_lists = [], []
        strides = (ctypes.c_size_t * n)()
        outs = (ctypes.c_void_p * n)()
        out_strides = (ctypes.c_size_t * n)()
        self.out_sizes = []
        for i, st in enumerate(stacks):
            descs[i] = stack_desc(st.width, st.height, len(st.frames), st.roi, st.channels, contrast_window,
                                  st.aligned, frames_per_batch, level_storage)
            fl = (ctypes.c_void_p * len(st.frames))(*[_ptr(f) for f in st.frames])
            frame_lists.append(fl)
            strides[i] = st.width * st.channels
            if st.poses is not None:
                pl = (_lib.FsPose * len(st.poses))(*[p.to_c() for p in st.poses])
            else:
                pl = None
            pose_lists.append(pl)
            outs[i] = _ptr(st.out)
            w = st.roi.width if (st.roi is not None and not st.aligned) else st.width
            h = st.roi.height if (st.roi is not None and not st.aligned) else st.height
            out_strides[i] = w * 3
            self.out_sizes.append((w, h))
        fptrs = (ctypes.POINTER(ctypes.c_void_p) * n)(*[ctypes.cast(f, ctypes.POINTER(ctypes.c_void_p))
                                                         for f in frame_lists])
        pptrs = (ctypes.POINTER(_lib.FsPose) * n)(*[ctypes.cast(p, ctypes.POINTER(_lib.FsPose)) if p is not None
                                                     else ctypes.POINTER(_lib.FsPose)() for p in pose_lists])
        any_pose = any(p is not None for p in pose_lists)
        h = ctypes.c_void_p()
        self._keep = (descs, frame_lists, pose_lists, strides, outs, out_strides, fptrs, pptrs, list(stacks))
        _check(L().fs_batch_create(ctx.handle, n, descs, fptrs, strides, pptrs if any_pose else None, outs,
                                   out_strides, lanes, pass2_mode, ctypes.byref(h)), ctx.handle)
        self.handle = h

    def run(self):
        _check(L().fs_batch_run(self.handle), self.ctx.handle)

    @property
    def uses_graph(self) -> bool:
        return bool(L().fs_batch_uses_graph(self.handle))

    def pass2_modes(self) -> List[str]:
        return [PASS2_MODES[L().fs_batch_pass2_mode(self.handle, i)] for i in range(len(self.out_sizes))]

    def close(self):
        if self.handle:
            L().fs_batch_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ precision form
STORAGE_F32 = 0   # pyramid levels stored in FP32 (the plain method)
STORAGE_F16 = 1   # levels stored in FP16, blends and accumulators in FP32
STORAGE_BF16 = 2  # levels stored in BF16, blends and accumulators in FP32
STORAGE_NAMES = {STORAGE_F32: "f32", STORAGE_F16: "f16", STORAGE_BF16: "bf16"}


def error_vs_reference(base: np.ndarray, ref_base: np.ndarray, out: Optional[np.ndarray] = None,
                       ref_out: Optional[np.ndarray] = None) -> dict:
    """Error of a fused result against a reference evaluation (the FP64
    oracle): max-abs and PSNR (peak 255) of the collapsed base before
    quantisation, in 8-bit units and in LSBs of a 16-bit output (x 257), and
    the largest u8 output difference when both outputs are given."""
    d = np.abs(np.asarray(base, np.float64) - np.asarray(ref_base, np.float64))
    mse = float(np.mean(d * d))
    r = {"max_abs": float(d.max()), "max_abs_lsb16": float(d.max() * 257.0),
         "psnr_db": float("inf") if mse == 0 else float(10.0 * np.log10(255.0 ** 2 / mse))}
    if out is not None and ref_out is not None:
        r["max_u8_diff"] = int(np.abs(out.astype(np.int16) - ref_out.astype(np.int16)).max())
    return r


# ------------------------------------------------------------------ synthetic
SCENE_SMALL = 0       # blur <= 3 px, shifts +-20 px, roll +-0.2 deg (1024x768-class stacks)
SCENE_PRODUCTION = 1  # blur <= 8 px, shifts +-60 px, roll +-0.3 deg (7952x5304-class stacks)


def synth_pose(seed: int, scene: int, width: int, height: int, frame: int, frame_count: int) -> ImagePose:
    p = _lib.FsPose()
    _check(L().fs_synth_pose(seed, scene, width, height, frame, frame_count, ctypes.byref(p)))
    return ImagePose.from_c(p)


def check_normalise(ctx: Context, w, n, out):
    """out = w / n elementwise (device float32 buffers of one length) as the
    split pyramid's level-0 blend divides: Markstein's refinement from n's
    correctly rounded reciprocal; for tests against the IEEE division."""
    count = int(w.numel())
    if int(n.numel()) != count or int(out.numel()) != count:
        raise FocusCudaError(2, "check_normalise: buffers of different lengths")
    _check(L().fs_check_normalise(ctx.handle, _ptr(w), _ptr(n), _ptr(out), count), ctx.handle)


def synth_frame_device(ctx: Context, seed: int, scene: int, width: int, height: int, frame: int, frame_count: int,
                       dst, dst_stride: int) -> ImagePose:
    p = _lib.FsPose()
    _check(L().fs_synth_frame_device(ctx.handle, seed, scene, width, height, frame, frame_count, _ptr(dst), dst_stride,
                                     ctypes.byref(p)), ctx.handle)
    return ImagePose.from_c(p)
