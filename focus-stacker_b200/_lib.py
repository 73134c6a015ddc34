"""ctypes binding of libfocuscuda.so (the C ABI in include/focuscuda.h).

The shared library is built in-tree (csrc/Makefile) and loaded from this
directory.  Importing does not need a GPU; calls that launch kernels fail
with FocusCudaError(FS_ERR_NO_DEVICE) when there is none.  There is no CPU
fallback: if the library is missing the import fails loudly.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfocuscuda.so")

FS_OK = 0
STATUS_NAMES = {
    0: "FS_OK", 1: "FS_ERR_INVALID", 2: "FS_ERR_OOM", 3: "FS_ERR_BUDGET", 4: "FS_ERR_CUDA",
    5: "FS_ERR_TIMEOUT", 6: "FS_ERR_STATE", 7: "FS_ERR_MISMATCH", 8: "FS_ERR_UNSUPPORTED",
    9: "FS_ERR_NO_DEVICE",
}

# Every function the header declares (checked by the CPU tests).
EXPORTED = (
    "fs_create", "fs_destroy", "fs_last_error", "fs_status_string", "fs_api_version", "fs_ctx_device_bytes",
    "fs_ctx_budget",
    "fs_ctx_synchronize", "fs_ctx_trim", "fs_ctx_reserve", "fs_ctx_set_budget", "fs_ctx_set_level_schedule", "fs_check_normalise", "fs_ctx_stream", "fs_ctx_launch_count", "fs_ctx_set_kernel_timing", "fs_ctx_kernel_stats",
    "fs_pose_default", "fs_compute_roi", "fs_inverse_map_points", "fs_forward_map_points", "fs_exact_expand_divisor",
    "fs_remap_frame", "fs_remap_frame_device", "fs_remap_frame16", "fs_remap_frame16_device",
    "fs_stack_begin", "fs_stack_add_frame", "fs_stack_add_frame_async", "fs_stack_add_frame_device", "fs_stack_finish",
    "fs_stack_finish_device", "fs_stack_finish_async", "fs_stack_wait", "fs_stack_set_base_output", "fs_stack_pass2_mode", "fs_stack_footprint", "fs_stack_mode_bytes", "fs_stack_begin_mode",
    "fs_stack_set_method", "fs_stack_set_frame_total", "fs_stack_end_pass1", "fs_stack_blend", "fs_stack_collapse", "fs_stack_buffer", "fs_stack_output_size", "fs_stack_destroy", "fs_fuse_stack",
    "fs_batch_create", "fs_batch_run", "fs_batch_stack_count", "fs_batch_pass2_mode", "fs_batch_uses_graph",
    "fs_batch_destroy",
    "fs_fuse_aligned_device_static", "fs_synth_frame_device", "fs_synth_pose",
    "fs_jpeg_info", "fs_decode_jpeg", "fs_stack_add_frame_jpeg",
)


class FsPose(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "yaw", "pitch", "roll", "hfov_delta", "trans_x", "trans_y", "trans_z", "translation_plane_yaw",
        "translation_plane_pitch", "radial_a", "radial_b", "radial_c", "center_shift_x", "center_shift_y",
        "base_hfov_degrees")]


class FsRect(ctypes.Structure):
    _fields_ = [("left", ctypes.c_int32), ("top", ctypes.c_int32), ("right", ctypes.c_int32),
                ("bottom", ctypes.c_int32)]


class FsStackDesc(ctypes.Structure):
    _fields_ = [
        ("src_width", ctypes.c_uint32), ("src_height", ctypes.c_uint32), ("has_roi", ctypes.c_int32),
        ("roi", FsRect), ("channels", ctypes.c_uint32), ("sample_bits", ctypes.c_uint32),
        ("frame_count", ctypes.c_uint32), ("contrast_window", ctypes.c_uint32),
        ("input_is_aligned", ctypes.c_int32), ("level_storage", ctypes.c_int32),
        ("frames_per_batch", ctypes.c_uint32),
    ]


FETCH_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p),
                            ctypes.POINTER(ctypes.c_size_t))

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libfocuscuda.so not found at {LIB_PATH}; build it with `make -C focus-stacker_b200/csrc` "
                "(or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        _bind(L)
        _lib = L
    return _lib


def _bind(L):
    P, vp, u32, i32, sz, u64 = ctypes.POINTER, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_size_t, ctypes.c_uint64
    ctx = vp
    L.fs_create.argtypes = [i32, u64, P(vp)]
    L.fs_destroy.argtypes = [ctx]
    L.fs_destroy.restype = None
    L.fs_last_error.argtypes = [ctx]
    L.fs_last_error.restype = ctypes.c_char_p
    L.fs_status_string.argtypes = [i32]
    L.fs_status_string.restype = ctypes.c_char_p
    L.fs_api_version.argtypes = []
    L.fs_ctx_device_bytes.argtypes = [ctx]
    L.fs_ctx_device_bytes.restype = u64
    L.fs_ctx_budget.argtypes = [ctx]
    L.fs_ctx_budget.restype = u64
    L.fs_ctx_synchronize.argtypes = [ctx]
    L.fs_ctx_trim.argtypes = [ctx]
    L.fs_ctx_reserve.argtypes = [ctx, u64]
    L.fs_ctx_set_budget.argtypes = [ctx, u64]
    L.fs_ctx_set_level_schedule.argtypes = [ctx, ctypes.c_uint32, ctypes.c_uint32]
    L.fs_check_normalise.argtypes = [ctx, vp, vp, vp, sz]
    L.fs_ctx_stream.argtypes = [ctx, P(vp)]
    L.fs_ctx_launch_count.argtypes = [ctx]
    L.fs_ctx_launch_count.restype = u64
    L.fs_ctx_set_kernel_timing.argtypes = [ctx, i32]
    L.fs_ctx_kernel_stats.argtypes = [ctx, ctypes.c_char_p, P(u64), P(ctypes.c_double)]
    L.fs_pose_default.argtypes = [P(FsPose)]
    L.fs_pose_default.restype = None
    L.fs_compute_roi.argtypes = [P(FsPose), P(u32), P(u32), P(ctypes.c_uint8), sz, P(FsRect), P(i32)]
    L.fs_inverse_map_points.argtypes = [P(FsPose), u32, u32, sz, P(ctypes.c_double), P(ctypes.c_double)]
    L.fs_forward_map_points.argtypes = [P(FsPose), u32, u32, sz, P(ctypes.c_double), P(ctypes.c_double)]
    L.fs_exact_expand_divisor.argtypes = [i32, i32, i32, i32]
    L.fs_exact_expand_divisor.restype = ctypes.c_float
    for f in (L.fs_remap_frame, L.fs_remap_frame_device, L.fs_remap_frame16, L.fs_remap_frame16_device):
        f.argtypes = [ctx, vp, sz, u32, u32, u32, P(FsPose), P(FsRect), vp, sz]
    L.fs_stack_begin.argtypes = [ctx, P(FsStackDesc), P(vp)]
    L.fs_stack_add_frame.argtypes = [vp, vp, sz, P(FsPose)]
    L.fs_stack_add_frame_async.argtypes = [vp, vp, sz, P(FsPose)]
    L.fs_stack_add_frame_device.argtypes = [vp, vp, sz, P(FsPose)]
    L.fs_stack_finish.argtypes = [vp, FETCH_CB, vp, vp, sz]
    L.fs_stack_finish_device.argtypes = [vp, FETCH_CB, vp, vp, sz]
    L.fs_stack_finish_async.argtypes = [vp, FETCH_CB, vp, vp, sz]
    L.fs_stack_wait.argtypes = [vp]
    L.fs_stack_output_size.argtypes = [vp, P(u32), P(u32)]
    L.fs_stack_set_base_output.argtypes = [vp, vp, sz]
    L.fs_stack_pass2_mode.argtypes = [vp]
    L.fs_stack_footprint.argtypes = [P(FsStackDesc), u64, i32, P(u64), P(i32)]
    L.fs_stack_mode_bytes.argtypes = [P(FsStackDesc), i32, i32, P(u64)]
    L.fs_stack_begin_mode.argtypes = [ctx, P(FsStackDesc), i32, P(vp)]
    L.fs_stack_set_method.argtypes = [vp, i32, ctypes.c_float]
    L.fs_stack_set_frame_total.argtypes = [vp, u32]
    L.fs_stack_end_pass1.argtypes = [vp]
    L.fs_stack_blend.argtypes = [vp, FETCH_CB, vp]
    L.fs_stack_collapse.argtypes = [vp, vp, sz, i32]
    L.fs_stack_buffer.argtypes = [vp, i32, u32, P(vp), P(u64), P(ctypes.c_int64), P(u32), P(u32)]
    L.fs_stack_destroy.argtypes = [vp]
    L.fs_fuse_stack.argtypes = [ctx, P(FsStackDesc), P(vp), P(sz), P(FsPose), vp, sz]
    L.fs_fuse_aligned_device_static.argtypes = [P(vp), P(sz), u32, u32, u32, u32, u32, vp, sz, vp,
                                                ctypes.c_char_p, sz]
    L.fs_batch_create.argtypes = [ctx, u32, P(FsStackDesc), P(P(vp)), P(sz), P(P(FsPose)), P(vp), P(sz), u32, i32,
                                  P(vp)]
    L.fs_batch_run.argtypes = [vp]
    L.fs_batch_stack_count.argtypes = [vp]
    L.fs_batch_pass2_mode.argtypes = [vp, u32]
    L.fs_batch_uses_graph.argtypes = [vp]
    L.fs_batch_destroy.argtypes = [vp]
    L.fs_synth_frame_device.argtypes = [ctx, u64, i32, u32, u32, u32, u32, vp, sz, P(FsPose)]
    L.fs_synth_pose.argtypes = [u64, i32, u32, u32, u32, u32, P(FsPose)]
    L.fs_jpeg_info.argtypes = [vp, sz, P(u32), P(u32)]
    L.fs_decode_jpeg.argtypes = [ctx, vp, sz, vp, sz, i32]
    L.fs_stack_add_frame_jpeg.argtypes = [vp, vp, sz, P(FsPose)]
