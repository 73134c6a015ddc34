// Shared host/device definitions of libfocuscuda: per-frame warp records and
// level geometry.
#pragma once

#include <stdint.h>
#include <stddef.h>

#ifdef __CUDACC__
#define FS_HD __host__ __device__ __forceinline__
#else
#define FS_HD inline
#endif

namespace fs {

// ------------------------------------------------------------- warp record
// Per-frame map from an output (aligned, ROI-relative) pixel (X, Y) to its
// source-frame sample position, composed on the host in FP64.  With
// D = 1 + g*X + h*Y:
//     x_src = X + (a*X + b*Y + c - X*(g*X + h*Y)) / D
//     y_src = Y + (d*X + e*Y + f - Y*(g*X + h*Y)) / D
// i.e. the homography [[1+a, b, c], [d, 1+e, f], [g, h, 1]] written as a
// displacement so that FP64 evaluation keeps ~1e-13 px absolute accuracy.
// For lens poses the same map yields the radial-space point (before the
// source centre); the radial inverse then runs per pixel.
enum WarpKind : int32_t {
  WARP_HOMOGRAPHY = 0,   // basic rectilinear, translation without radial, shift only
  WARP_RADIAL = 1,       // homography to radial space + Newton radial inverse (lens poses)
  WARP_ALIGNED = 2,      // input already aligned: identity, no resampling
};

struct Warp {
  int32_t kind;
  int32_t guard;          // 1: the denominator may reach <= 0 inside the ROI (every pixel takes the exact path)
  int32_t behind_is_void; // 1: D <= 0 gives an empty sample (basic chain); 0: |D| < eps gives empty (lens path)
  float tie_band;         // fast FP32 sampler: values within this of a .5 rounding boundary take the
                          // exact path (from the map's error bound; kernels use at least 2.5e-4)
  double a, b, c, d, e, f, g, h;  // displacement-form homography coefficients
  // radial inverse (WARP_RADIAL): src = centre + undistort(radial point)
  double src_cx, src_cy;
  double radial_a, radial_b, radial_c, radial_inv_norm;
  double eps_den;         // |D| threshold mirroring the reference's 1e-12 on its own scale
};

// ---------------------------------------------------------- level geometry
FS_HD uint32_t next_level_size(uint32_t v) { return v > 1 ? (v + 1) / 2 : 1; }
FS_HD uint32_t level_count(uint32_t w, uint32_t h) {
  uint32_t levels = 1;
  while (w > 1 || h > 1) {
    w = next_level_size(w);
    h = next_level_size(h);
    ++levels;
  }
  return levels;
}
static const uint32_t kExactExpandMaxDim = 512;  // below or at this size the no-wrap expand is used

}  // namespace fs
