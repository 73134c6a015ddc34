"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is a line-by-line C++ restatement of the reference's remap and
pyramid-contrast fusion (see focus_oracle.cpp for per-function citations).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module, as the checker; the shipped library never calls it.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_libs = {}


def build() -> str:
    """Compile the oracle with its Makefile (g++, strict IEEE)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _native_path() -> str:
    """The -march=native build for this host's CPU (one directory per CPU
    model and flag set, built on first use): the timed CPU baseline."""
    key = ""
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith(("model name", "flags")):
                    key += line
                if line.strip() == "":
                    break
    except OSError:
        key = "unknown"
    tag = hashlib.sha1(key.encode()).hexdigest()[:12]
    out = os.path.join(_HERE, "_build", "native-" + tag)
    subprocess.run(["make", "-s", "-C", _HERE, "native", "NATIVE_OUT=" + out], check=True)
    return os.path.join(out, "liboracle.so")


def lib(native: bool = False):
    """The oracle library: the portable build (parity checks), or with
    native=True the -march=native build for this host (timed baselines; the
    same strict-IEEE arithmetic, so the same results)."""
    key = "native" if native else "portable"
    if key not in _libs:
        if native:
            path = _native_path()
        else:
            path = _LIB_PATH
            if not os.path.exists(path):
                build()
        L = ctypes.CDLL(path)
        _bind(L)
        _libs[key] = L
    return _libs[key]


POSE_FIELDS = (
    "yaw", "pitch", "roll", "hfov_delta", "trans_x", "trans_y", "trans_z",
    "translation_plane_yaw", "translation_plane_pitch", "radial_a", "radial_b",
    "radial_c", "center_shift_x", "center_shift_y", "base_hfov_degrees",
)


class _Pose(ctypes.Structure):
    _fields_ = [("v", ctypes.c_double * 15)]


def pose_array(poses) -> ctypes.Array:
    """poses: sequence of dicts / objects with ImagePose fields (defaults as the reference)."""
    arr = (_Pose * max(1, len(poses)))()
    for i, p in enumerate(poses):
        arr[i] = _Pose((ctypes.c_double * 15)(*pose_values(p)))
    return arr


def pose_values(p) -> list:
    defaults = dict.fromkeys(POSE_FIELDS, 0.0)
    defaults["base_hfov_degrees"] = 50.0
    if p is None:
        p = {}
    if not isinstance(p, dict):
        p = {k: getattr(p, k) for k in POSE_FIELDS}
    d = dict(defaults)
    d.update(p)
    return [float(d[k]) for k in POSE_FIELDS]


def _bind(L):
    P = ctypes.POINTER
    dp, fp, vp = P(ctypes.c_double), P(ctypes.c_float), ctypes.c_void_p
    u32, i32, sz = ctypes.c_uint32, ctypes.c_int, ctypes.c_size_t
    L.oracle_inverse_point.argtypes = [P(_Pose), u32, u32, ctypes.c_double, ctypes.c_double, dp, dp]
    L.oracle_forward_point.argtypes = [P(_Pose), u32, u32, ctypes.c_double, ctypes.c_double, dp, dp]
    L.oracle_compute_roi.argtypes = [P(_Pose), P(u32), P(u32), P(ctypes.c_uint8), sz, P(ctypes.c_int32)]
    L.oracle_compute_roi.restype = i32
    L.oracle_remap.argtypes = [vp, u32, u32, i32, i32, P(_Pose), P(ctypes.c_int32), i32, vp]
    L.oracle_weight_map.argtypes = [vp, u32, u32, i32, i32, u32, i32, fp]
    L.oracle_fill_average.argtypes = [vp, u32, u32, i32, i32, fp]
    L.oracle_sample_stddev.argtypes = [ctypes.c_double, ctypes.c_double, u32]
    L.oracle_sample_stddev.restype = ctypes.c_float
    L.oracle_normalize_weights.argtypes = [fp, fp, sz, fp, sz]
    L.oracle_level_count.argtypes = [u32, u32]
    L.oracle_level_count.restype = sz
    for name in ("oracle_reduce_rgb_with_support", "oracle_reduce_scalar_with_support"):
        getattr(L, name).argtypes = [u32, u32, fp, fp, fp, fp]
    L.oracle_reduce_rgb_plain.argtypes = [u32, u32, fp, fp]
    L.oracle_expand_rgb.argtypes = [u32, u32, u32, u32, fp, fp]
    L.oracle_fuse_aligned.argtypes = [P(vp), sz, u32, u32, i32, i32, u32, i32, i32, vp, dp]
    L.oracle_fuse_aligned.restype = i32
    L.oracle_stack_fuse.argtypes = [P(vp), sz, u32, u32, i32, P(_Pose), P(ctypes.c_int32), u32, i32, i32, vp, dp]
    L.oracle_stack_fuse.restype = i32
    L.oracle_update_winners.argtypes = [vp, sz, i32, i32, fp, fp, vp]
    L.oracle_update_winners.restype = None
    L.oracle_stack_fuse_hybrid.argtypes = [P(vp), sz, u32, u32, i32, P(_Pose), P(ctypes.c_int32), u32, i32, u32, u32,
                                           ctypes.c_float, vp, dp, vp]
    L.oracle_stack_fuse_hybrid.restype = i32
    L.oracle_hybrid_merge.argtypes = [vp, vp, u32, u32, i32, u32, u32, ctypes.c_float, i32, vp, dp]
    L.oracle_hybrid_merge.restype = None
    L.oracle_pyramid_floats.argtypes = [u32, u32]
    L.oracle_pyramid_floats.restype = sz
    L.oracle_pyramid_accumulate.argtypes = [vp, u32, u32, i32, i32, fp, fp, fp, i32]
    L.oracle_pyramid_accumulate.restype = None
    L.oracle_pyramid_collapse.argtypes = [fp, u32, u32, i32, vp, dp, i32]
    L.oracle_pyramid_collapse.restype = None
    L.oracle_synth_pose.argtypes = [ctypes.c_uint64, i32, u32, u32, u32, u32, P(_Pose)]
    L.oracle_synth_render.argtypes = [ctypes.c_uint64, i32, u32, u32, u32, u32, u32, u32, vp, sz, i32]


def _ptr(a: np.ndarray, ctype=None):
    if ctype is None:
        return ctypes.c_void_p(a.ctypes.data)
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def inverse_point(pose, width, height, x, y):
    sx, sy = ctypes.c_double(), ctypes.c_double()
    lib().oracle_inverse_point(pose_array([pose]), width, height, x, y, ctypes.byref(sx), ctypes.byref(sy))
    return sx.value, sy.value


def forward_point(pose, width, height, x, y):
    ox, oy = ctypes.c_double(), ctypes.c_double()
    lib().oracle_forward_point(pose_array([pose]), width, height, x, y, ctypes.byref(ox), ctypes.byref(oy))
    return ox.value, oy.value


def compute_roi(poses, widths, heights, active=None):
    n = len(poses)
    w = np.ascontiguousarray(widths, dtype=np.uint32)
    h = np.ascontiguousarray(heights, dtype=np.uint32)
    a = np.ones(n, np.uint8) if active is None else np.ascontiguousarray(active, dtype=np.uint8)
    out = np.zeros(4, np.int32)
    ok = lib().oracle_compute_roi(pose_array(poses), _ptr(w, ctypes.c_uint32), _ptr(h, ctypes.c_uint32),
                                  _ptr(a, ctypes.c_uint8), n, _ptr(out, ctypes.c_int32))
    return tuple(int(v) for v in out) if ok else None


def remap(src: np.ndarray, pose, roi=None, jobs=1) -> np.ndarray:
    """src: HxW (1 channel) or HxWxC uint8/uint16.  Returns ROI-sized HxWx(C+1)."""
    src = np.ascontiguousarray(src)
    h, w = src.shape[:2]
    ch = 1 if src.ndim == 2 else src.shape[2]
    bits = 8 if src.dtype == np.uint8 else 16
    if roi is None:
        roi = (0, 0, w, h)
    ow, oh = roi[2] - roi[0], roi[3] - roi[1]
    out = np.zeros((oh, ow, ch + 1), src.dtype)
    r = np.asarray(roi, np.int32)
    lib().oracle_remap(_ptr(src), w, h, ch, bits, pose_array([pose]), _ptr(r, ctypes.c_int32), jobs, _ptr(out))
    return out


def weight_map(img: np.ndarray, window=5, jobs=1) -> np.ndarray:
    img = np.ascontiguousarray(img)
    h, w, c = img.shape
    out = np.zeros((h, w), np.float32)
    lib().oracle_weight_map(_ptr(img), w, h, c - 3, 8 if img.dtype == np.uint8 else 16, window, jobs,
                            _ptr(out, ctypes.c_float))
    return out


def fill_average(img: np.ndarray) -> np.ndarray:
    img = np.ascontiguousarray(img)
    h, w, c = img.shape
    out = np.zeros((h, w), np.float32)
    lib().oracle_fill_average(_ptr(img), w, h, c - 3, 8 if img.dtype == np.uint8 else 16, _ptr(out, ctypes.c_float))
    return out


def sample_stddev(s, ss, n):
    return lib().oracle_sample_stddev(s, ss, n)


def normalize_weights(w, norm, total_images):
    w = np.ascontiguousarray(w, np.float32)
    norm = np.ascontiguousarray(norm, np.float32)
    out = np.zeros_like(w)
    lib().oracle_normalize_weights(_ptr(w, ctypes.c_float), _ptr(norm, ctypes.c_float), total_images,
                                   _ptr(out, ctypes.c_float), w.size)
    return out


def level_count(w, h):
    return int(lib().oracle_level_count(w, h))


def next_level_size(v):
    return (v + 1) // 2 if v > 1 else 1


def reduce_with_support(src: np.ndarray, support: np.ndarray):
    src = np.ascontiguousarray(src, np.float32)
    support = np.ascontiguousarray(support, np.float32)
    sh, sw = support.shape
    dh, dw = next_level_size(sh), next_level_size(sw)
    rgb = src.ndim == 3
    dst = np.zeros((dh, dw, 3) if rgb else (dh, dw), np.float32)
    dsup = np.zeros((dh, dw), np.float32)
    f = lib().oracle_reduce_rgb_with_support if rgb else lib().oracle_reduce_scalar_with_support
    f(sw, sh, _ptr(src, ctypes.c_float), _ptr(support, ctypes.c_float), _ptr(dst, ctypes.c_float),
      _ptr(dsup, ctypes.c_float))
    return dst, dsup


def reduce_rgb_plain(src: np.ndarray):
    src = np.ascontiguousarray(src, np.float32)
    sh, sw = src.shape[:2]
    dst = np.zeros((next_level_size(sh), next_level_size(sw), 3), np.float32)
    lib().oracle_reduce_rgb_plain(sw, sh, _ptr(src, ctypes.c_float), _ptr(dst, ctypes.c_float))
    return dst


def expand_rgb(src: np.ndarray, dst_w: int, dst_h: int):
    src = np.ascontiguousarray(src, np.float32)
    sh, sw = src.shape[:2]
    dst = np.zeros((dst_h, dst_w, 3), np.float32)
    lib().oracle_expand_rgb(dst_w, dst_h, sw, sh, _ptr(src, ctypes.c_float), _ptr(dst, ctypes.c_float))
    return dst


def fuse_aligned(frames, window=5, jobs=1, precision=32, want_base=False):
    """frames: list of HxWx3 or HxWx4 uint8/uint16 aligned images."""
    frames = [np.ascontiguousarray(f) for f in frames]
    h, w, c = frames[0].shape
    bits = 8 if frames[0].dtype == np.uint8 else 16
    ptrs = (ctypes.c_void_p * len(frames))(*[f.ctypes.data for f in frames])
    out = np.zeros((h, w, 3), frames[0].dtype)
    base = np.zeros((h, w, 3), np.float64) if want_base else None
    rc = lib().oracle_fuse_aligned(ptrs, len(frames), w, h, c - 3, bits, window, jobs, precision, _ptr(out),
                                   _ptr(base, ctypes.c_double) if want_base else None)
    if rc != 0:
        raise RuntimeError("oracle_fuse_aligned failed")
    return (out, base) if want_base else out


def stack_fuse(sources, poses, roi=None, window=5, jobs=1, precision=32, want_base=False, native=False):
    """sources: list of HxWx3 uint8/uint16 frames; poses: list of pose dicts.
    native=True runs the -march=native build (timed baselines)."""
    sources = [np.ascontiguousarray(s) for s in sources]
    h, w = sources[0].shape[:2]
    bits = 8 if sources[0].dtype == np.uint8 else 16
    if roi is None:
        roi = (0, 0, w, h)
    ow, oh = roi[2] - roi[0], roi[3] - roi[1]
    ptrs = (ctypes.c_void_p * len(sources))(*[s.ctypes.data for s in sources])
    out = np.zeros((oh, ow, 3), sources[0].dtype)
    base = np.zeros((oh, ow, 3), np.float64) if want_base else None
    r = np.asarray(roi, np.int32)
    rc = lib(native).oracle_stack_fuse(ptrs, len(sources), w, h, bits, pose_array(poses), _ptr(r, ctypes.c_int32),
                                       window,
                                 jobs, precision, _ptr(out), _ptr(base, ctypes.c_double) if want_base else None)
    if rc != 0:
        raise RuntimeError("oracle_stack_fuse failed")
    return (out, base) if want_base else out


def update_winners(image: np.ndarray, weights: np.ndarray, best: np.ndarray, out: np.ndarray):
    """blend.updateWinners on one image (HxWx3 or HxWx4, uint8/uint16):
    best (float32) and out (HxWx3) are updated in place."""
    image = np.ascontiguousarray(image)
    weights = np.ascontiguousarray(weights, np.float32)
    assert best.dtype == np.float32 and best.flags.c_contiguous and out.flags.c_contiguous
    h, w, c = image.shape
    lib().oracle_update_winners(_ptr(image), h * w, c - 3, 8 if image.dtype == np.uint8 else 16,
                                _ptr(weights, ctypes.c_float), _ptr(best, ctypes.c_float), _ptr(out))


HYBRID_HARD_LEVEL_START, HYBRID_HARD_LEVEL_COUNT, HYBRID_SHARPNESS = 2, 4, 0.35


def stack_fuse_hybrid(sources, poses, roi=None, window=5, jobs=1, mix=HYBRID_SHARPNESS,
                      hard_start=HYBRID_HARD_LEVEL_START, hard_count=HYBRID_HARD_LEVEL_COUNT, want_base=False,
                      want_hard=False):
    """hybrid-pyramid-contrast of a stack (src/stack/pipeline.zig:177-236)."""
    sources = [np.ascontiguousarray(s) for s in sources]
    h, w = sources[0].shape[:2]
    bits = 8 if sources[0].dtype == np.uint8 else 16
    if roi is None:
        roi = (0, 0, w, h)
    ow, oh = roi[2] - roi[0], roi[3] - roi[1]
    ptrs = (ctypes.c_void_p * len(sources))(*[s.ctypes.data for s in sources])
    out = np.zeros((oh, ow, 3), sources[0].dtype)
    base = np.zeros((oh, ow, 3), np.float64)
    hard = np.zeros((oh, ow, 3), sources[0].dtype)
    r = np.asarray(roi, np.int32)
    rc = lib().oracle_stack_fuse_hybrid(ptrs, len(sources), w, h, bits, pose_array(poses), _ptr(r, ctypes.c_int32),
                                        window, jobs, hard_start, hard_count, mix, _ptr(out),
                                        _ptr(base, ctypes.c_double), _ptr(hard))
    if rc != 0:
        raise RuntimeError("oracle_stack_fuse_hybrid failed")
    res = [out]
    if want_base:
        res.append(base)
    if want_hard:
        res.append(hard)
    return tuple(res) if len(res) > 1 else out


def hybrid_merge(soft: np.ndarray, hard: np.ndarray, mix=HYBRID_SHARPNESS, hard_start=HYBRID_HARD_LEVEL_START,
                 hard_count=HYBRID_HARD_LEVEL_COUNT, jobs=1):
    """mergeHybridImages of two HxWx3 images; returns (image, base)."""
    soft, hard = np.ascontiguousarray(soft), np.ascontiguousarray(hard)
    h, w = soft.shape[:2]
    out = np.zeros_like(soft)
    base = np.zeros((h, w, 3), np.float64)
    lib().oracle_hybrid_merge(_ptr(soft), _ptr(hard), w, h, 8 if soft.dtype == np.uint8 else 16, hard_start,
                              hard_count, mix, jobs, _ptr(out), _ptr(base, ctypes.c_double))
    return out, base


def pyramid_floats(width, height) -> int:
    """Floats of an accumulator pyramid (all levels, interleaved RGB)."""
    return int(lib().oracle_pyramid_floats(width, height))


def pyramid_accumulate(frame: np.ndarray, normalized_mask: np.ndarray, union_support: np.ndarray, acc: np.ndarray,
                       jobs=1):
    """Pass 2 of one aligned frame (HxWx3/4) into acc (float32, in place)."""
    frame = np.ascontiguousarray(frame)
    h, w, c = frame.shape
    m = np.ascontiguousarray(normalized_mask, np.float32)
    u = np.ascontiguousarray(union_support, np.float32)
    assert acc.dtype == np.float32 and acc.flags.c_contiguous and acc.size == pyramid_floats(w, h)
    lib().oracle_pyramid_accumulate(_ptr(frame), w, h, c - 3, 8 if frame.dtype == np.uint8 else 16,
                                    _ptr(m, ctypes.c_float), _ptr(u, ctypes.c_float), _ptr(acc, ctypes.c_float), jobs)


def pyramid_collapse(acc: np.ndarray, width, height, sample_bits=8, jobs=1):
    """Collapse and quantise an accumulator pyramid; returns (image, base)."""
    acc = np.ascontiguousarray(acc, np.float32)
    out = np.zeros((height, width, 3), np.uint8 if sample_bits == 8 else np.uint16)
    base = np.zeros((height, width, 3), np.float64)
    lib().oracle_pyramid_collapse(_ptr(acc, ctypes.c_float), width, height, sample_bits, _ptr(out),
                                  _ptr(base, ctypes.c_double), jobs)
    return out, base


# ------------------------------------------------------ synthetic stacks
SCENE_SMALL, SCENE_PRODUCTION = 0, 1


def synth_pose(seed, scene, width, height, frame, frame_count) -> dict:
    """Pose of synthetic frame `frame` as a dict of ImagePose fields (the
    device generator's draws)."""
    p = (_Pose * 1)()
    lib().oracle_synth_pose(seed, scene, width, height, frame, frame_count, p)
    return dict(zip(POSE_FIELDS, list(p[0].v)))


def synth_frame(seed, scene, width, height, frame, frame_count, rows=None, jobs=1, native=False):
    """Synthetic frame `frame` rendered on the CPU (HxWx3 uint8).  rows =
    (first, count) renders only those rows; the others stay zero and untouched
    (their pages are never written)."""
    img = np.zeros((height, width, 3), np.uint8)
    r0, n = (0, height) if rows is None else rows
    lib(native).oracle_synth_render(seed, scene, width, height, frame, frame_count, max(0, r0), max(0, n),
                                    _ptr(img), width * 3, jobs)
    return img
