// Device-side remap of one output pixel: bilinear sample with support alpha,
// bit-exact with the reference's f64 sampler (src/remap.zig:710-839,
// 939-970) for 8-bit RGB / gray sources.
//
// Precision scheme (no FP64 on the device):
//  * the source position is the host-composed projective map evaluated in
//    double-float (two FP32) as a displacement from the output pixel, good to
//    ~1e-12 px (fs_common.h, Warp);
//  * FAST path: per 8x4 pixel block a double-float anchor is formed once, and
//    each pixel's position offset from the anchor is a small FP32 rational
//    (error < 1e-7 px).  The FP32 bilinear value is then within 1e-4 of the
//    exact one; when every channel's value is farther than kTieBand from a
//    .5 rounding boundary and the 4 taps lie at least one pixel inside the
//    frame, the result is certain and equals the reference's;
//  * EXACT path (edge band, near-ties, guarded or lens poses): everything in
//    double-float, with the reference's edge rules (soft support, alpha =
//    round(support * 255), empty sample when support <= 0).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fs_common.h"

namespace fs {

// Source image for the remap: interleaved u8, `ch` = 1 or 3 samples/pixel.
struct SrcImage {
  const uint8_t* px;
  int64_t pitch;  // bytes per row
  int32_t w, h;
  int32_t ch;
};

static constexpr float kTieBand = 2.5e-4f;

// Pixel record produced by the remap: R | G << 8 | B << 16 | A << 24.
__device__ __forceinline__ uint32_t pack_rgba(uint32_t r, uint32_t g, uint32_t b, uint32_t a) {
  return r | (g << 8) | (b << 16) | (a << 24);
}

__device__ __forceinline__ void load_rgb(const SrcImage& s, int x, int y, float v[3]) {
  const uint8_t* p = s.px + (int64_t)y * s.pitch + (int64_t)x * s.ch;
  if (s.ch == 3) {
    v[0] = (float)__ldg(p);
    v[1] = (float)__ldg(p + 1);
    v[2] = (float)__ldg(p + 2);
  } else {
    v[0] = (float)__ldg(p);
    v[1] = v[0];
    v[2] = v[0];
  }
}

// Taps of the fast path as biased floats 2^23 + v (exact, one OR): the
// differences of two taps are exact without removing the bias.
__device__ __forceinline__ void load_rgb_biased(const SrcImage& s, int x, int y, float v[3]) {
  const uint8_t* p = s.px + (int64_t)y * s.pitch + (int64_t)x * s.ch;
  if (s.ch == 3) {
    v[0] = __uint_as_float(0x4B000000u | (uint32_t)__ldg(p));
    v[1] = __uint_as_float(0x4B000000u | (uint32_t)__ldg(p + 1));
    v[2] = __uint_as_float(0x4B000000u | (uint32_t)__ldg(p + 2));
  } else {
    v[0] = __uint_as_float(0x4B000000u | (uint32_t)__ldg(p));
    v[1] = v[0];
    v[2] = v[0];
  }
}

// Block anchor for the fast path.
struct Anchor {
  int32_t ix, iy;        // integer part of the anchor's source position
  float fxh, fxl, fyh, fyl;  // fractional part (double-float)
  float am1x, bx, ay, bm1y, gam, eta;
};

// Displacement (source - output) of output pixel (X, Y), double-float.
// Returns false when the denominator is outside the map's valid domain.
__device__ __forceinline__ bool warp_disp(const Warp& w, float X, float Y, dfl* dx, dfl* dy, dfl* Dout) {
  dfl dD = df_add(df_mul_f(w.g, X), df_mul_f(w.h, Y));
  dfl D = df_add_f(dD, 1.0f);
  if (Dout) *Dout = D;
  if (w.behind_is_void) {
    if (!(D.hi > 0.0f)) return false;
  } else {
    if (fabsf(D.hi) < (float)w.eps_den) return false;
  }
  dfl nx = df_add(df_add(df_mul_f(w.a, X), df_mul_f(w.b, Y)), w.c);
  nx = df_sub(nx, df_mul_f(dD, X));
  dfl ny = df_add(df_add(df_mul_f(w.d, X), df_mul_f(w.e, Y)), w.f);
  ny = df_sub(ny, df_mul_f(dD, Y));
  *dx = df_div(nx, D);
  *dy = df_div(ny, D);
  return true;
}

// Block anchor broadcast from lane `src` of the warp.
__device__ __forceinline__ Anchor shfl_anchor(const Anchor& a, int src) {
  const unsigned full = 0xffffffffu;
  Anchor o;
  o.ix = __shfl_sync(full, a.ix, src);
  o.iy = __shfl_sync(full, a.iy, src);
  o.fxh = __shfl_sync(full, a.fxh, src);
  o.fxl = __shfl_sync(full, a.fxl, src);
  o.fyh = __shfl_sync(full, a.fyh, src);
  o.fyl = __shfl_sync(full, a.fyl, src);
  o.am1x = __shfl_sync(full, a.am1x, src);
  o.bx = __shfl_sync(full, a.bx, src);
  o.ay = __shfl_sync(full, a.ay, src);
  o.bm1y = __shfl_sync(full, a.bm1y, src);
  o.gam = __shfl_sync(full, a.gam, src);
  o.eta = __shfl_sync(full, a.eta, src);
  return o;
}

__device__ __forceinline__ Anchor make_anchor(const Warp& w, int X, int Y, bool* ok) {
  Anchor a = {};
  dfl dx, dy, D;
  float Xf = (float)X, Yf = (float)Y;
  *ok = warp_disp(w, Xf, Yf, &dx, &dy, &D);
  if (!*ok) return a;
  float flx = df_floor(dx), fly = df_floor(dy);
  a.ix = X + (int)flx;
  a.iy = Y + (int)fly;
  dfl fx = df_add_f(dx, -flx), fy = df_add_f(dy, -fly);
  a.fxh = fx.hi; a.fxl = fx.lo;
  a.fyh = fy.hi; a.fyl = fy.lo;
  // x(X+du, Y+dv) - x_a - du = ((alpha-1) du + beta dv - du (gam du + eta dv)) / (1 + gam du + eta dv)
  // with alpha = (h00 - x_a h20) / D, beta = (h01 - x_a h21) / D, gam = h20 / D, eta = h21 / D,
  // h00 = 1 + a, h01 = b, h20 = g, h21 = h and x_a = X + dx.
  dfl xa = df_add_f(dx, Xf), ya = df_add_f(dy, Yf);
  dfl dDa = df_sub(D, df_make(1.0f));
  dfl am1 = df_div(df_sub(df_sub(w.a, df_mul(xa, w.g)), dDa), D);
  dfl bx = df_div(df_sub(w.b, df_mul(xa, w.h)), D);
  dfl ay = df_div(df_sub(w.d, df_mul(ya, w.g)), D);
  dfl bm1 = df_div(df_sub(df_sub(w.e, df_mul(ya, w.h)), dDa), D);
  a.am1x = am1.hi; a.bx = bx.hi; a.ay = ay.hi; a.bm1y = bm1.hi;
  a.gam = df_div(w.g, D).hi;
  a.eta = df_div(w.h, D).hi;
  return a;
}

// Round-half-away of value / support decided exactly in double-float.
__device__ __forceinline__ uint32_t df_round_ratio(dfl value, dfl support) {
  float q = value.hi / support.hi;
  float k = floorf(q);
  dfl t = df_sub(value, df_mul_f(support, k + 0.5f));
  float r = df_sign(t) >= 0 ? k + 1.0f : k;
  r = fminf(fmaxf(r, 0.0f), 255.0f);
  return (uint32_t)r;
}

// Newton radial inverse with the reference's stopping rules, double-float
// (src/remap.zig:755-786).
static __device__ dfl df_sqrt(dfl a) {
  if (a.hi <= 0.0f) return df_make(0.0f);
  float s = sqrtf(a.hi);
  dfl s2 = df_two_prod(s, s);
  dfl r = df_sub(a, s2);
  float c = r.hi / (2.0f * s);
  return df_fast_two_sum(s, c);
}

static __device__ void radial_inverse_df(const Warp& w, dfl dx, dfl dy, dfl* ox, dfl* oy) {
  dfl q = df_sqrt(df_add(df_mul(dx, dx), df_mul(dy, dy)));
  if (q.hi < 1e-12f) {
    *ox = dx;
    *oy = dy;
    return;
  }
  dfl r = q;
  for (int it = 0; it < 6; ++it) {
    dfl r2 = df_mul(df_mul(r, r), w.radial_inv_norm);
    dfl r4 = df_mul(r2, r2);
    dfl fac = df_add(df_add(df_add_f(df_mul(w.radial_a, r2), 1.0f), df_mul(w.radial_b, r4)),
                     df_mul(df_mul(w.radial_c, r4), r2));
    dfl der = df_add(df_add(w.radial_a, df_mul_f(df_mul(w.radial_b, r2), 2.0f)), df_mul_f(df_mul(w.radial_c, r4), 3.0f));
    dfl f = df_sub(df_mul(r, fac), q);
    if (fabsf(f.hi) <= 1e-9f) break;
    dfl dfd = df_add(fac, df_mul(df_mul_f(df_mul(df_mul(r, r), w.radial_inv_norm), 2.0f), der));
    if (fabsf(dfd.hi) < 1e-12f) break;
    r = df_sub(r, df_div(f, dfd));
    if (r.hi < 0.0f) r = df_make(0.0f);
  }
  dfl s = df_div(r, q);
  *ox = df_mul(dx, s);
  *oy = df_mul(dy, s);
}

// Exact sample of output pixel (X, Y) (ROI-relative), all decisions in
// double-float.  Follows samplePixelBilinearU8 (src/remap.zig:710-753).
static __device__ __noinline__ uint32_t sample_exact(const Warp& w, const SrcImage& s, int X, int Y) {
  dfl dx, dy;
  float Xf = (float)X, Yf = (float)Y;
  if (!warp_disp(w, Xf, Yf, &dx, &dy, nullptr)) return 0u;
  int x0, y0;
  dfl fx, fy;
  if (w.kind == WARP_RADIAL) {
    dfl px = df_sub(df_add_f(dx, Xf), w.src_cx), py = df_sub(df_add_f(dy, Yf), w.src_cy);
    dfl ux, uy;
    radial_inverse_df(w, px, py, &ux, &uy);
    dfl sx = df_add(w.src_cx, ux), sy = df_add(w.src_cy, uy);
    float flx = df_floor(sx), fly = df_floor(sy);
    if (!(fabsf(flx) < 1e8f && fabsf(fly) < 1e8f)) return 0u;
    x0 = (int)flx;
    y0 = (int)fly;
    fx = df_add_f(sx, -flx);
    fy = df_add_f(sy, -fly);
  } else {
    float flx = df_floor(dx), fly = df_floor(dy);
    if (!(fabsf(flx) < 1e8f && fabsf(fly) < 1e8f)) return 0u;
    x0 = X + (int)flx;
    y0 = Y + (int)fly;
    fx = df_add_f(dx, -flx);
    fy = df_add_f(dy, -fly);
  }
  dfl one = df_make(1.0f);
  dfl omfx = df_sub(one, fx), omfy = df_sub(one, fy);
  dfl wt[4] = {df_mul(omfx, omfy), df_mul(fx, omfy), df_mul(omfx, fy), df_mul(fx, fy)};
  int tx[4] = {x0, x0 + 1, x0, x0 + 1};
  int ty[4] = {y0, y0, y0 + 1, y0 + 1};
  bool inb[4];
  bool all_in = true;
  for (int i = 0; i < 4; ++i) {
    inb[i] = tx[i] >= 0 && ty[i] >= 0 && tx[i] < s.w && ty[i] < s.h;
    all_in = all_in && inb[i];
  }
  dfl support = df_make(0.0f);
  for (int i = 0; i < 4; ++i)
    if (inb[i]) support = df_add(support, wt[i]);
  if (df_sign(support) <= 0) return 0u;
  dfl val[3] = {df_make(0.0f), df_make(0.0f), df_make(0.0f)};
  for (int i = 0; i < 4; ++i) {
    if (!inb[i]) continue;
    float v[3];
    load_rgb(s, tx[i], ty[i], v);
    for (int c = 0; c < 3; ++c) val[c] = df_add(val[c], df_mul_f(wt[i], v[c]));
  }
  uint32_t out[3];
  for (int c = 0; c < 3; ++c) out[c] = df_round_ratio(val[c], support);
  uint32_t alpha;
  if (all_in) {
    alpha = 255u;
  } else {
    alpha = df_round_ratio(df_mul_f(support, 255.0f), df_make(1.0f));
  }
  return pack_rgba(out[0], out[1], out[2], alpha);
}

// Fast path only: returns false (leaving *out untouched) when the exact
// path must decide the sample.
__device__ __forceinline__ bool sample_try(const SrcImage& s, const Anchor& a, int du, int dv, uint32_t* out) {
  float fdu = (float)du, fdv = (float)dv;
  float gd = fmaf(a.gam, fdu, a.eta * fdv);
  float den = 1.0f + gd;
  float nx = fmaf(a.am1x, fdu, a.bx * fdv) - fdu * gd;
  float ny = fmaf(a.ay, fdu, a.bm1y * fdv) - fdv * gd;
  float rd = __fdividef(1.0f, den);
  float tx = a.fxh + fmaf(nx, rd, a.fxl);
  float ty = a.fyh + fmaf(ny, rd, a.fyl);
  float flx = floorf(tx), fly = floorf(ty);
  int x0 = a.ix + du + (int)flx;
  int y0 = a.iy + dv + (int)fly;
  float fx = tx - flx, fy = ty - fly;
  if (x0 < 1 || y0 < 1 || x0 > s.w - 3 || y0 > s.h - 3) return false;
  float v00[3], v10[3], v01[3], v11[3];
  load_rgb_biased(s, x0, y0, v00);
  load_rgb_biased(s, x0 + 1, y0, v10);
  load_rgb_biased(s, x0, y0 + 1, v01);
  load_rgb_biased(s, x0 + 1, y0 + 1, v11);
  float fxy = fx * fy;
  uint32_t o[3];
  bool tie = false;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float d10 = v10[c] - v00[c], d01 = v01[c] - v00[c], d11 = (v11[c] - v10[c]) - d01;
    float v = fmaf(fx, d10, v00[c] - 8388608.0f);
    v = fmaf(fy, d01, v);
    v = fmaf(fxy, d11, v);
    float k = floorf(v);
    float fr = v - k;
    tie = tie || fabsf(fr - 0.5f) < kTieBand;
    float r = fr > 0.5f ? k + 1.0f : k;
    o[c] = (uint32_t)fminf(fmaxf(r, 0.0f), 255.0f);
  }
  if (tie) return false;
  *out = pack_rgba(o[0], o[1], o[2], 255u);
  return true;
}

// Sample output pixel (X, Y) = anchor pixel + (du, dv).  Falls back to the
// exact path when the fast path cannot certify the result.
__device__ __forceinline__ uint32_t sample_fast(const Warp& w, const SrcImage& s, const Anchor& a, int du, int dv,
                                                int X, int Y) {
  float fdu = (float)du, fdv = (float)dv;
  float gd = fmaf(a.gam, fdu, a.eta * fdv);
  float den = 1.0f + gd;
  float nx = fmaf(a.am1x, fdu, a.bx * fdv) - fdu * gd;
  float ny = fmaf(a.ay, fdu, a.bm1y * fdv) - fdv * gd;
  float rd = __fdividef(1.0f, den);
  float tx = a.fxh + fmaf(nx, rd, a.fxl);
  float ty = a.fyh + fmaf(ny, rd, a.fyl);
  float flx = floorf(tx), fly = floorf(ty);
  int x0 = a.ix + du + (int)flx;
  int y0 = a.iy + dv + (int)fly;
  float fx = tx - flx, fy = ty - fly;
  // taps at least one pixel inside on every side: the floor decision then
  // cannot change which sampler the reference takes
  if (x0 < 1 || y0 < 1 || x0 > s.w - 3 || y0 > s.h - 3) return sample_exact(w, s, X, Y);
  float v00[3], v10[3], v01[3], v11[3];
  load_rgb_biased(s, x0, y0, v00);
  load_rgb_biased(s, x0 + 1, y0, v10);
  load_rgb_biased(s, x0, y0 + 1, v01);
  load_rgb_biased(s, x0 + 1, y0 + 1, v11);
  float fxy = fx * fy;
  uint32_t o[3];
  bool tie = false;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float d10 = v10[c] - v00[c], d01 = v01[c] - v00[c], d11 = (v11[c] - v10[c]) - d01;
    float v = fmaf(fx, d10, v00[c] - 8388608.0f);
    v = fmaf(fy, d01, v);
    v = fmaf(fxy, d11, v);
    float k = floorf(v);
    float fr = v - k;
    tie = tie || fabsf(fr - 0.5f) < kTieBand;
    float r = fr > 0.5f ? k + 1.0f : k;
    o[c] = (uint32_t)fminf(fmaxf(r, 0.0f), 255.0f);
  }
  if (tie) return sample_exact(w, s, X, Y);
  return pack_rgba(o[0], o[1], o[2], 255u);
}

}  // namespace fs
