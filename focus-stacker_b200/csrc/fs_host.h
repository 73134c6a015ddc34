// Host-side declarations shared by the C-ABI and the kernel launchers.
#pragma once

#include <stdint.h>

#include "../../include/focuscuda.h"
#include "fs_common.h"

namespace fs {

// Compose the per-frame output->source map (FP64, once per frame).
bool compose_warp(const fs_pose& pose, uint32_t src_w, uint32_t src_h, const fs_rect& roi, Warp* out,
                  const char** why);
// FP64 evaluation of the composed map at one aligned-frame point.
void inverse_map_point_f64(const fs_pose& pose, uint32_t w, uint32_t h, double x, double y, double* sx, double* sy);
// Forward map source -> aligned frame (the reference's transformPoint).
void forward_map_point(const fs_pose& pose, uint32_t w, uint32_t h, double x, double y, double* ox, double* oy);
// Common-overlap ROI (FP64), false when empty.
bool compute_roi(const fs_pose* poses, const uint32_t* widths, const uint32_t* heights, const uint8_t* active,
                 size_t n, fs_rect* out);

}  // namespace fs
