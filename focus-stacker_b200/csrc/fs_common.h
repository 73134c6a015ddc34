// Shared host/device definitions of libfocuscuda: per-frame warp records,
// double-float (pairs of FP32) arithmetic, level geometry.
#pragma once

#include <stdint.h>
#include <stddef.h>

#ifdef __CUDACC__
#define FS_HD __host__ __device__ __forceinline__
#define FS_DF __device__ __forceinline__
#else
#define FS_HD inline
#define FS_DF inline
#endif

namespace fs {

// ------------------------------------------------------------ double-float
// An unevaluated sum hi + lo of two FP32 numbers (|lo| <= ulp(hi)/2): about
// 48 significant bits from FP32 arithmetic.  Used by the remap for the
// sample coordinate and for the rare exact tie-breaks; no FP64 on the device.
struct dfl {
  float hi, lo;
};

#ifdef __CUDACC__
#define FS_ADD(a, b) __fadd_rn((a), (b))
#define FS_SUB(a, b) __fsub_rn((a), (b))
#define FS_MUL(a, b) __fmul_rn((a), (b))
#define FS_FMA(a, b, c) __fmaf_rn((a), (b), (c))
#else
#define FS_ADD(a, b) ((a) + (b))
#define FS_SUB(a, b) ((a) - (b))
#define FS_MUL(a, b) ((a) * (b))
#define FS_FMA(a, b, c) fmaf((a), (b), (c))
#endif

FS_DF dfl df_make(float v) { return {v, 0.0f}; }
// Knuth two-sum: s + e == a + b exactly.
FS_DF dfl df_two_sum(float a, float b) {
  float s = FS_ADD(a, b);
  float bb = FS_SUB(s, a);
  float e = FS_ADD(FS_SUB(a, FS_SUB(s, bb)), FS_SUB(b, bb));
  return {s, e};
}
// Dekker fast two-sum, requires |a| >= |b|.
FS_DF dfl df_fast_two_sum(float a, float b) {
  float s = FS_ADD(a, b);
  float e = FS_SUB(b, FS_SUB(s, a));
  return {s, e};
}
FS_DF dfl df_two_prod(float a, float b) {
  float p = FS_MUL(a, b);
  float e = FS_FMA(a, b, -p);
  return {p, e};
}
FS_DF dfl df_add(dfl a, dfl b) {
  dfl s = df_two_sum(a.hi, b.hi);
  dfl t = df_two_sum(a.lo, b.lo);
  s.lo = FS_ADD(s.lo, t.hi);
  s = df_fast_two_sum(s.hi, s.lo);
  s.lo = FS_ADD(s.lo, t.lo);
  return df_fast_two_sum(s.hi, s.lo);
}
FS_DF dfl df_neg(dfl a) { return {-a.hi, -a.lo}; }
FS_DF dfl df_sub(dfl a, dfl b) { return df_add(a, df_neg(b)); }
FS_DF dfl df_add_f(dfl a, float b) {
  dfl s = df_two_sum(a.hi, b);
  s.lo = FS_ADD(s.lo, a.lo);
  return df_fast_two_sum(s.hi, s.lo);
}
FS_DF dfl df_mul(dfl a, dfl b) {
  dfl p = df_two_prod(a.hi, b.hi);
  p.lo = FS_FMA(a.hi, b.lo, p.lo);
  p.lo = FS_FMA(a.lo, b.hi, p.lo);
  return df_fast_two_sum(p.hi, p.lo);
}
FS_DF dfl df_mul_f(dfl a, float b) {
  dfl p = df_two_prod(a.hi, b);
  p.lo = FS_FMA(a.lo, b, p.lo);
  return df_fast_two_sum(p.hi, p.lo);
}
#ifdef __CUDACC__
#define FS_FDIV(a, b) __fdividef((a), (b))
#else
#define FS_FDIV(a, b) ((a) / (b))
#endif
// a / b: an approximate FP32 quotient (a few ulp) refined by two exact
// remainder corrections, which is what carries the ~2^-46 accuracy.
FS_DF dfl df_div(dfl a, dfl b) {
  float rb = FS_FDIV(1.0f, b.hi);
  float q1 = FS_MUL(a.hi, rb);
  dfl r = df_sub(a, df_mul_f(b, q1));
  float q2 = FS_MUL(r.hi, rb);
  r = df_sub(r, df_mul_f(b, q2));
  float q3 = FS_MUL(r.hi, rb);
  dfl q = df_fast_two_sum(q1, q2);
  return df_add_f(q, q3);
}
// sign of a (a.hi carries the sign unless a.hi == 0).
FS_DF int df_sign(dfl a) { return a.hi > 0.0f ? 1 : (a.hi < 0.0f ? -1 : (a.lo > 0.0f ? 1 : (a.lo < 0.0f ? -1 : 0))); }
// floor of a double-float, returned as float (exact integer).
FS_DF float df_floor(dfl a) {
  float f = floorf(a.hi);
  if (f == a.hi && a.lo < 0.0f) f -= 1.0f;
  return f;
}

// ------------------------------------------------------------- warp record
// Per-frame map from an output (aligned, ROI-relative) pixel (X, Y) to its
// source-frame sample position, composed on the host in FP64.  With
// D = 1 + g*X + h*Y:
//     x_src = X + (a*X + b*Y + c - X*(g*X + h*Y)) / D
//     y_src = Y + (d*X + e*Y + f - Y*(g*X + h*Y)) / D
// i.e. the homography [[1+a, b, c], [d, 1+e, f], [g, h, 1]] written as a
// displacement so that double-float keeps ~1e-12 px absolute accuracy.
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
  int32_t pad0;
  dfl a, b, c, d, e, f, g, h;  // displacement-form homography coefficients
  // radial inverse (WARP_RADIAL): src = centre + undistort(radial point)
  dfl src_cx, src_cy;
  dfl radial_a, radial_b, radial_c, radial_inv_norm;
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
