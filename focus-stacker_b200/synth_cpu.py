"""CPU rendering of synthetic focus stacks with the recipe of the device
generator (csrc/synth.cu): 64 sinusoids with amplitudes U(5, 30), random
orientation and phase, spatial frequencies in [0.05, 1.2] rad/px on an even
grid of w^2, per-pixel Gaussian blur sigma = min(|d - z_k| * s, cap) applied
analytically, contrast gain 0.28, per-channel gain/offset, N(0, 4^2) noise,
rounded to u8.  Poses come from the library's host generator (fs_synth_pose)
and each source pixel is rendered at its forward-mapped scene point.

Used where frames must be made without a GPU (the CPU baseline); pixel values
are not bit-identical to the device renderer's, the distributions are the same.
"""
from __future__ import annotations

import math

import numpy as np

from .api import ImagePose, forward_map_points, synth_pose

_BLUR = {0: (3.0, 3.0), 1: (8.0, 8.0)}


def synth_frame_cpu(seed: int, scene: int, width: int, height: int, frame: int, frame_count: int):
    pose: ImagePose = synth_pose(seed, scene, width, height, frame, frame_count)
    rng = np.random.default_rng(seed)
    n = 64
    wmin, wmax = 0.05, 1.2
    w = np.sqrt(wmin ** 2 + (wmax ** 2 - wmin ** 2) * np.arange(n) / (n - 1))
    amp = rng.uniform(5.0, 30.0, n)
    theta = rng.uniform(0.0, math.pi, n)
    phase = rng.uniform(0.0, 2 * math.pi, n)
    order = rng.permutation(n)
    amp, theta, phase = amp[order], theta[order], phase[order]
    dfx, dfy = rng.uniform(0.3, 2.0, 6), rng.uniform(0.3, 2.0, 6)
    dang, dph, da = rng.uniform(0, 2 * math.pi, 6), rng.uniform(0, 1, 6), rng.uniform(0.5, 1.0, 6)
    gain, offset = rng.uniform(0.9, 1.1, 3), rng.uniform(-10, 10, 3)
    scale, cap = _BLUR[scene]
    z = frame / (frame_count - 1) if frame_count > 1 else 0.5

    ys, xs = np.mgrid[0:height, 0:width]
    pts = np.stack([xs.ravel(), ys.ravel()], 1).astype(np.float64)
    X, Y = forward_map_points(pose, width, height, pts).T
    d = np.zeros_like(X)
    for t in range(6):
        d += da[t] * np.cos(2 * math.pi * (dfx[t] * math.cos(dang[t]) * X / width +
                                           dfy[t] * math.sin(dang[t]) * Y / height + dph[t]))
    d = 0.5 + 0.5 * d / da.sum()
    sigma = np.minimum(np.abs(d - z) * scale, cap)
    s2 = (sigma * sigma).astype(np.float32)
    # attenuation exp(-s^2 w_i^2 / 2): w_i^2 is an even grid, so consecutive
    # components differ by one factor per pixel
    att = np.exp(-0.5 * s2 * np.float32(w[0] ** 2))
    rat = np.exp(-0.5 * s2 * np.float32(w[1] ** 2 - w[0] ** 2))
    X32, Y32 = X.astype(np.float32), Y.astype(np.float32)
    tex = np.zeros_like(X32)
    ph = np.empty_like(X32)
    for i in range(n):
        np.multiply(X32, np.float32(w[i] * math.cos(theta[i])), out=ph)
        ph += Y32 * np.float32(w[i] * math.sin(theta[i]))
        ph += np.float32(phase[i])
        np.sin(ph, out=ph)
        ph *= att
        tex += np.float32(amp[i]) * ph
        att *= rat
    noise = rng.normal(0.0, 4.0, (X.size, 3)).astype(np.float32)
    out = 128.0 + offset[None, :] + gain[None, :] * 0.28 * tex[:, None] + noise
    img = np.clip(np.rint(out), 0, 255).astype(np.uint8).reshape(height, width, 3)
    return img, pose
