"""B200 (sm_100a) implementation of the focus-stacker remap + pyramid-contrast
fusion hot path: a C-ABI shared library (libfocuscuda.so, csrc/) and its
host-side mirror of the reference's operator interface (api.py).

The directory name carries a hyphen, so load it with load_package() (or
importlib) under the module name `focus_stacker_b200`.
"""
from . import _lib  # noqa: F401
from . import serving  # noqa: F401
from . import autotune  # noqa: F401
from . import sharded  # noqa: F401
from .api import (  # noqa: F401
    Context, FocusCudaError, ImagePose, Method, PyramidContrastStack, Rect, SCENE_PRODUCTION, SCENE_SMALL,
    STORAGE_BF16, STORAGE_F16, STORAGE_F32, STORAGE_NAMES, compute_common_overlap_roi, error_vs_reference,
    BUFFER_ACCUMULATOR, BUFFER_HARD, BUFFER_UNION, BUFFER_WEIGHT_SUM, BatchStack, FUSION_METHODS, HYBRID_SHARPNESS,
    decode_jpeg, decode_jpeg_device, jpeg_info, DeviceBuffer, StackBatch, stack_desc,
    stack_footprint, stack_mode_bytes, exact_expand_divisor, forward_map_points, fuse_aligned_images, fuse_remapped_images,
    inverse_map_points, parse_method, parse_window_size, remap_rigid_image, remap_rigid_image_device,
    synth_frame_device, synth_pose, check_normalise,
)
