// Device-side remap of one output pixel: bilinear sample with support alpha,
// bit-exact with the reference's f64 sampler (src/remap.zig:710-839,
// 939-970) for 8-bit RGB / gray sources.
//
// Precision scheme:
//  * the source position is the host-composed projective map evaluated in
//    FP64 as a displacement from the output pixel, good to ~1e-13 px
//    (fs_common.h, Warp);
//  * FAST path: per 8x4 pixel block an FP64 anchor is formed once (split
//    into two FP32 words), and each pixel's position offset from the anchor
//    is a small FP32 rational (error < 1e-7 px for near-identity maps).  The
//    FP32 bilinear value is then within 1e-4 of the exact one; when every
//    channel's value is farther than the frame's tie band from a .5 rounding
//    boundary and the 4 taps lie at least one pixel inside the frame, the
//    result is certain and equals the reference's.  The band is kTieBand or
//    more: the host widens it from the map's error bound (Warp::tie_band);
//    maps far from the identity take wider bands and the exact path more often;
//  * EXACT path (edge band, near-ties, guarded or lens poses): the
//    reference's f64 sampler op for op (products and sums rounded one by one,
//    no fused multiply-add), with its edge rules (soft support, alpha =
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

// Block anchor for the fast path (48 bytes: three 16-byte shared loads).
struct __align__(16) Anchor {
  int32_t ix, iy;        // integer part of the anchor's source position
  float fxh, fxl, fyh, fyl;  // fractional part (double-float)
  float am1x, bx, ay, bm1y, gam, eta;
};

// Displacement (source - output) of output pixel (X, Y), FP64.  Returns
// false when the denominator is outside the map's valid domain.
__device__ __forceinline__ bool warp_disp(const Warp& w, double X, double Y, double* dx, double* dy, double* Dout) {
  const double dD = fma(w.g, X, w.h * Y);
  const double D = dD + 1.0;
  if (Dout) *Dout = D;
  if (w.behind_is_void) {
    if (!(D > 0.0)) return false;
  } else {
    if (fabs(D) < w.eps_den) return false;
  }
  const double nx = fma(w.a, X, fma(w.b, Y, w.c)) - dD * X;
  const double ny = fma(w.d, X, fma(w.e, Y, w.f)) - dD * Y;
  const double rD = 1.0 / D;  // one division; x rD is within an ulp of / D
  *dx = nx * rD;
  *dy = ny * rD;
  return true;
}

__device__ __forceinline__ Anchor make_anchor(const Warp& w, int X, int Y, bool* ok) {
  Anchor a = {};
  double dx, dy, D;
  const double Xd = (double)X, Yd = (double)Y;
  *ok = warp_disp(w, Xd, Yd, &dx, &dy, &D);
  if (!*ok) return a;
  const double flx = floor(dx), fly = floor(dy);
  if (!(fabs(flx) < 1e8 && fabs(fly) < 1e8)) {
    *ok = false;
    return a;
  }
  a.ix = X + (int)flx;
  a.iy = Y + (int)fly;
  const double fx = dx - flx, fy = dy - fly;  // exact
  a.fxh = (float)fx;
  a.fxl = (float)(fx - (double)a.fxh);
  a.fyh = (float)fy;
  a.fyl = (float)(fy - (double)a.fyh);
  // x(X+du, Y+dv) - x_a - du = ((alpha-1) du + beta dv - du (gam du + eta dv)) / (1 + gam du + eta dv)
  // with alpha = (h00 - x_a h20) / D, beta = (h01 - x_a h21) / D, gam = h20 / D, eta = h21 / D,
  // h00 = 1 + a, h01 = b, h20 = g, h21 = h and x_a = X + dx.
  const double xa = dx + Xd, ya = dy + Yd, dDa = D - 1.0, rD = 1.0 / D;
  a.am1x = (float)((w.a - xa * w.g - dDa) * rD);
  a.bx = (float)((w.b - xa * w.h) * rD);
  a.ay = (float)((w.d - ya * w.g) * rD);
  a.bm1y = (float)((w.e - ya * w.h - dDa) * rD);
  a.gam = (float)(w.g * rD);
  a.eta = (float)(w.h * rD);
  return a;
}

// Newton radial inverse with the reference's stopping rules and operation
// order (src/remap.zig:755-786): returns the undistorted offset.
static __device__ void radial_inverse(const Warp& w, double dx, double dy, double* ox, double* oy) {
  const double q = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
  if (q < 1e-12) {
    *ox = dx;
    *oy = dy;
    return;
  }
  double r = q;
  for (int it = 0; it < 6; ++it) {
    const double r2 = __dmul_rn(__dmul_rn(r, r), w.radial_inv_norm);
    const double r4 = __dmul_rn(r2, r2);
    const double fac = __dadd_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(w.radial_a, r2)), __dmul_rn(w.radial_b, r4)),
                                 __dmul_rn(__dmul_rn(w.radial_c, r4), r2));
    const double fd = __dadd_rn(__dadd_rn(w.radial_a, __dmul_rn(__dmul_rn(2.0, w.radial_b), r2)),
                                __dmul_rn(__dmul_rn(3.0, w.radial_c), r4));
    const double f = __dsub_rn(__dmul_rn(r, fac), q);
    if (fabs(f) <= 1e-9) break;
    const double df = __dadd_rn(fac, __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(2.0, r), r), w.radial_inv_norm), fd));
    if (fabs(df) < 1e-12) break;
    r = __dsub_rn(r, __ddiv_rn(f, df));
    r = fmax(r, 0.0);
  }
  const double sc = __ddiv_rn(r, q);
  *ox = __dmul_rn(dx, sc);
  *oy = __dmul_rn(dy, sc);
}

// Exact sample of output pixel (X, Y) (ROI-relative): the reference's f64
// bilinear sampler (samplePixelBilinearU8, src/remap.zig:710-753, interior
// :788-839, soft edge :939-994) with products and sums rounded one at a time.
static __device__ __noinline__ uint32_t sample_exact(const Warp& w, const SrcImage& s, int X, int Y) {
  double dx, dy;
  const double Xd = (double)X, Yd = (double)Y;
  if (!warp_disp(w, Xd, Yd, &dx, &dy, nullptr)) return 0u;
  int x0, y0;
  double fx, fy;
  if (w.kind == WARP_RADIAL) {
    double ux, uy;
    radial_inverse(w, __dsub_rn(dx + Xd, w.src_cx), __dsub_rn(dy + Yd, w.src_cy), &ux, &uy);
    const double sx = __dadd_rn(w.src_cx, ux), sy = __dadd_rn(w.src_cy, uy);
    const double flx = floor(sx), fly = floor(sy);
    if (!(fabs(flx) < 1e8 && fabs(fly) < 1e8)) return 0u;
    x0 = (int)flx;
    y0 = (int)fly;
    fx = sx - flx;
    fy = sy - fly;
  } else {
    const double flx = floor(dx), fly = floor(dy);
    if (!(fabs(flx) < 1e8 && fabs(fly) < 1e8)) return 0u;
    x0 = X + (int)flx;
    y0 = Y + (int)fly;
    fx = dx - flx;
    fy = dy - fly;
  }
  const double omfx = __dsub_rn(1.0, fx), omfy = __dsub_rn(1.0, fy);
  const double wt[4] = {__dmul_rn(omfx, omfy), __dmul_rn(fx, omfy), __dmul_rn(omfx, fy), __dmul_rn(fx, fy)};
  const int tx[4] = {x0, x0 + 1, x0, x0 + 1};
  const int ty[4] = {y0, y0, y0 + 1, y0 + 1};
  bool inb[4];
  bool all_in = true;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    inb[i] = tx[i] >= 0 && ty[i] >= 0 && tx[i] < s.w && ty[i] < s.h;
    all_in = all_in && inb[i];
  }
  double support = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (inb[i]) support = __dadd_rn(support, wt[i]);
  if (!(support > 0.0)) return 0u;
  double val[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (!inb[i]) continue;
    float v[3];
    load_rgb(s, tx[i], ty[i], v);
#pragma unroll
    for (int c = 0; c < 3; ++c) val[c] = __dadd_rn(val[c], __dmul_rn((double)v[c], wt[i]));
  }
  uint32_t out[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    // value / 1 is the value: skip the division when the weights sum to 1
    const double q = support == 1.0 ? val[c] : __ddiv_rn(val[c], support);
    out[c] = (uint32_t)fmin(fmax(round(q), 0.0), 255.0);
  }
  const uint32_t alpha = all_in ? 255u : (uint32_t)fmin(fmax(round(__dmul_rn(support, 255.0)), 0.0), 255.0);
  return pack_rgba(out[0], out[1], out[2], alpha);
}

// floor of v (|v| < 2^22) and its integer, without the float-to-int
// conversion unit: the nearest integer from adding and removing 1.5 * 2^23,
// minus one where that rounded up.
__device__ __forceinline__ float floor_small(float v, int* iv) {
  const float t = __fadd_rn(v, 12582912.0f);
  const float r = __fsub_rn(t, 12582912.0f);
  const bool up = r > v;
  *iv = (__float_as_int(t) - 0x4B400000) - (up ? 1 : 0);
  return up ? __fsub_rn(r, 1.0f) : r;
}

// Nearest integer of v (|v| < 2^22), clamped to 0..255, by adding and
// removing 1.5 * 2^23 (no float-to-int conversion), and the distance |v - r|:
// a value farther than 0.5 - kTieBand from r lies within kTieBand of a .5
// rounding boundary, where the FP32 evaluation cannot decide the reference's
// half-away rounding.  Away from those boundaries nearest rounding is it.
__device__ __forceinline__ uint32_t round_near_u8(float v, float* dist) {
  const float t = __fadd_rn(v, 12582912.0f);
  *dist = fabsf(__fsub_rn(v, __fsub_rn(t, 12582912.0f)));
  const int r = __float_as_int(t) - 0x4B400000;
  return (uint32_t)min(max(r, 0), 255);
}

// A frame's source for the fast sampler, held in registers for the whole
// region (CH = 3: RGB, 1: gray; 0: read at run time from `ch`).
struct TapSrc {
  const uint8_t* px;
  uint32_t pitch;  // bytes per row
  uint32_t xm, ym;  // fast taps need 1 <= x0 <= w - 3: (unsigned)(x0 - 1) <= w - 4 (w, h >= 4)
  int32_t ch;
  float lim;        // 0.5 - tie band
};

__device__ __forceinline__ TapSrc tap_src(const SrcImage& s, float tie_band) {
  TapSrc t;
  t.px = s.px;
  t.pitch = (uint32_t)s.pitch;
  t.xm = (uint32_t)(s.w - 4);
  t.ym = (uint32_t)(s.h - 4);
  t.ch = s.ch;
  t.lim = 0.5f - fmaxf(tie_band, kTieBand);
  return t;
}

// Support flag of a 16-bit contrast word (gray sum R + G + B in bits 0..14).
static constexpr uint32_t kSupportFlag = 1u << 15;

// Contrast word of a supported sample from its three channel floats
// 1.5 * 2^23 + c: gray sum R + G + B with the support flag.
__device__ __forceinline__ uint32_t biased_contrast_word(float r, float g, float b) {
  return __float_as_uint(r) + __float_as_uint(g) + __float_as_uint(b) + (kSupportFlag - 3u * 0x4B400000u);
}

// Fast path only: returns false (leaving *out untouched) when the exact path
// must decide the sample.  On success *out is the packed sample (alpha 255)
// and *kw its contrast word.  The source fields sit in registers (TapSrc),
// the tap addresses are one 32 x 32 -> 64-bit multiply-add per row and the
// taps are byte loads at immediate offsets from the two row pointers.
template <int CH>
__device__ __forceinline__ bool sample_try(const TapSrc& s, const Anchor& a, float fdu, float fdv, int du, int dv,
                                           uint32_t* out, uint32_t* kw) {
  const float gd = fmaf(a.gam, fdu, a.eta * fdv);
  const float rd = __fdividef(1.0f, 1.0f + gd);
  const float nx = fmaf(a.am1x, fdu, a.bx * fdv) - fdu * gd;
  const float ny = fmaf(a.ay, fdu, a.bm1y * fdv) - fdv * gd;
  const float tx = a.fxh + fmaf(nx, rd, a.fxl);
  const float ty = a.fyh + fmaf(ny, rd, a.fyl);
  int ixf, iyf;
  const float flx = floor_small(tx, &ixf), fly = floor_small(ty, &iyf);
  const int x0 = a.ix + du + ixf;
  const int y0 = a.iy + dv + iyf;
  // taps at least one pixel inside on every side: the floor decision then
  // cannot change which sampler the reference takes
  if ((uint32_t)(x0 - 1) > s.xm || (uint32_t)(y0 - 1) > s.ym) return false;
  const float fx = tx - flx, fy = ty - fly;
  const int ch = CH ? CH : s.ch;
  const uint8_t* r0 = s.px + ((uint64_t)(uint32_t)y0 * s.pitch + (uint32_t)(x0 * ch));
  const uint8_t* r1 = r0 + s.pitch;
  const float fxy = fx * fy;
  const float2 m1 = make_float2(-1.0f, -1.0f);
  const float2 M = make_float2(12582912.0f, 12582912.0f);
  auto bf = [](uint8_t v) { return __uint_as_float(0x4B000000u | (uint32_t)v); };
  if (CH == 1 || (CH == 0 && ch == 1)) {
    // gray: one channel, replicated
    const float v00 = bf(__ldg(r0)), v10 = bf(__ldg(r0 + 1)), v01 = bf(__ldg(r1)), v11 = bf(__ldg(r1 + 1));
    const float e10 = v10 - v00, e01 = v01 - v00, e11 = (v11 - v10) - e01;
    float v = fmaf(fx, e10, v00 - 8388608.0f);
    v = fmaf(fy, e01, v);
    v = fmaf(fxy, e11, v);
    const float t = __fadd_rn(v, 12582912.0f);
    const float d = __fsub_rn(v, __fsub_rn(t, 12582912.0f));
    if (fabsf(d) > s.lim) return false;
    const uint32_t g = __float_as_uint(t) & 255u;
    *out = g * 0x010101u | 0xFF000000u;
    *kw = 3u * g | kSupportFlag;
    return true;
  }
  const float2 a00 = make_float2(bf(__ldg(r0)), bf(__ldg(r0 + 1)));
  const float2 a10 = make_float2(bf(__ldg(r0 + ch)), bf(__ldg(r0 + ch + 1)));
  const float2 a01 = make_float2(bf(__ldg(r1)), bf(__ldg(r1 + 1)));
  const float2 a11 = make_float2(bf(__ldg(r1 + ch)), bf(__ldg(r1 + ch + 1)));
  const float b00 = bf(__ldg(r0 + 2)), b10 = bf(__ldg(r0 + ch + 2));
  const float b01 = bf(__ldg(r1 + 2)), b11 = bf(__ldg(r1 + ch + 2));
  // red and green as FP32 pairs (each lane of a pair rounds exactly like the
  // scalar operation: a - b is fma(b, -1, a)), blue alone
  const float2 d10 = __ffma2_rn(a00, m1, a10), d01 = __ffma2_rn(a00, m1, a01);
  const float2 d11 = __ffma2_rn(d01, m1, __ffma2_rn(a10, m1, a11));
  float2 v = __fadd2_rn(a00, make_float2(-8388608.0f, -8388608.0f));
  v = __ffma2_rn(make_float2(fx, fx), d10, v);
  v = __ffma2_rn(make_float2(fy, fy), d01, v);
  v = __ffma2_rn(make_float2(fxy, fxy), d11, v);
  const float e10 = b10 - b00, e01 = b01 - b00, e11 = (b11 - b10) - e01;
  float vb = fmaf(fx, e10, b00 - 8388608.0f);
  vb = fmaf(fy, e01, vb);
  vb = fmaf(fxy, e11, vb);
  // nearest integers by adding and removing 1.5 * 2^23: t's low byte is the
  // integer (a bilinear value of bytes lies in [0, 255] up to ~1e-4)
  const float2 t = __fadd2_rn(v, M);
  const float2 dl = __ffma2_rn(__fadd2_rn(t, make_float2(-12582912.0f, -12582912.0f)), m1, v);
  const float tb = __fadd_rn(vb, 12582912.0f);
  const float db = __fsub_rn(vb, __fsub_rn(tb, 12582912.0f));
  const float dmax = fmaxf(fmaxf(fabsf(dl.x), fabsf(dl.y)), fabsf(db));
  if (dmax > s.lim) return false;
  const uint32_t rg = __byte_perm(__float_as_uint(t.x), __float_as_uint(t.y), 0x0040u);
  *out = __byte_perm(rg, __float_as_uint(tb), 0x0410u) | 0xFF000000u;
  *kw = biased_contrast_word(t.x, t.y, tb);
  return true;
}

// Block anchor of the tile sampler: the integer position pre-biased so that
// one three-input add of the rounded-down float's bits gives x0 - 1 (see
// sample_tile), the rest as in Anchor.
struct __align__(16) TileAnchor {
  int32_t kx, ky;  // ix - 1 - 0x4B400000, iy - 1 - 0x4B400000; kx == kNoTileAnchor: none
  float fxh, fxl, fyh, fyl;
  float am1x, bx, ay, bm1y, gam, eta;
};
static constexpr int32_t kNoTileAnchor = INT32_MIN;  // |ix| < 1e8 keeps kx far from it

__device__ __forceinline__ TileAnchor tile_anchor(const Anchor& a) {
  TileAnchor t;
  t.kx = (int32_t)((uint32_t)a.ix - 1u - 0x4B400000u);
  t.ky = (int32_t)((uint32_t)a.iy - 1u - 0x4B400000u);
  t.fxh = a.fxh;
  t.fxl = a.fxl;
  t.fyh = a.fyh;
  t.fyl = a.fyl;
  t.am1x = a.am1x;
  t.bx = a.bx;
  t.ay = a.ay;
  t.bm1y = a.bm1y;
  t.gam = a.gam;
  t.eta = a.eta;
  return t;
}

// The fast sampler of the tile kernel, the same decision as sample_try with
// fewer operations and no branches (so that the loads of neighbouring
// samples overlap): floor(t) from one round-down add of 1.5 * 2^23 (its bits
// minus 0x4B400000 are the integer, |t| < 2^22), the taps' bounds as two
// unsigned compares of x0 - 1 and y0 - 1 against w - 4 and h - 4, 32-bit tap
// offsets from `org` (the frame's pixel (1, 1); frames below 4 GiB; a sample
// that fails the bounds reads the taps at `org` and is discarded).  `lim` is
// 0.5 - the frame's tie band.  Returns whether *out is decided.
template <int CH>
__device__ __forceinline__ bool sample_tile(const uint8_t* org, uint32_t pitch, uint32_t xm, uint32_t ym, float lim,
                                            const TileAnchor& a, float fdu, float fdv, int du, int dv,
                                            uint32_t* out) {
  const float gd = fmaf(a.gam, fdu, a.eta * fdv);
  const float rd = __fdividef(1.0f, 1.0f + gd);
  const float nx = fmaf(a.am1x, fdu, a.bx * fdv) - fdu * gd;
  const float ny = fmaf(a.ay, fdu, a.bm1y * fdv) - fdv * gd;
  const float tx = a.fxh + fmaf(nx, rd, a.fxl);
  const float ty = a.fyh + fmaf(ny, rd, a.fyl);
  const float sx = __fadd_rd(tx, 12582912.0f), sy = __fadd_rd(ty, 12582912.0f);
  const uint32_t xm1 = __float_as_uint(sx) + (uint32_t)a.kx + (uint32_t)du;  // x0 - 1
  const uint32_t ym1 = __float_as_uint(sy) + (uint32_t)a.ky + (uint32_t)dv;  // y0 - 1
  // taps at least one pixel inside on every side: the floor decision then
  // cannot change which sampler the reference takes
  bool ok = a.kx != kNoTileAnchor && xm1 <= xm && ym1 <= ym;
  const float fx = tx - (sx - 12582912.0f), fy = ty - (sy - 12582912.0f);
  const uint32_t o0 = ok ? ym1 * pitch + xm1 * (uint32_t)CH : 0u;
  const uint8_t* r0 = org + o0;
  const uint8_t* r1 = org + (o0 + pitch);
  const float fxy = fx * fy;
  // taps as biased floats 2^23 + v (one OR each): differences are exact
  // without removing the bias, which only the first tap's value drops
  auto bf = [](uint8_t v) { return __uint_as_float(0x4B000000u | (uint32_t)v); };
  if (CH == 1) {
    const float v00 = bf(__ldg(r0)), v10 = bf(__ldg(r0 + 1)), v01 = bf(__ldg(r1)), v11 = bf(__ldg(r1 + 1));
    const float e10 = v10 - v00, e01 = v01 - v00, e11 = (v11 - v10) - e01;
    float v = fmaf(fx, e10, v00 - 8388608.0f);
    v = fmaf(fy, e01, v);
    v = fmaf(fxy, e11, v);
    const float t = __fadd_rn(v, 12582912.0f);
    ok = ok && fabsf(__fsub_rn(v, __fsub_rn(t, 12582912.0f))) <= lim;
    *out = (__float_as_uint(t) & 255u) * 0x010101u | 0xFF000000u;
    return ok;
  }
  const float2 m1 = make_float2(-1.0f, -1.0f);
  const float2 a00 = make_float2(bf(__ldg(r0)), bf(__ldg(r0 + 1)));
  const float2 a10 = make_float2(bf(__ldg(r0 + CH)), bf(__ldg(r0 + CH + 1)));
  const float2 a01 = make_float2(bf(__ldg(r1)), bf(__ldg(r1 + 1)));
  const float2 a11 = make_float2(bf(__ldg(r1 + CH)), bf(__ldg(r1 + CH + 1)));
  const float b00 = bf(__ldg(r0 + 2)), b10 = bf(__ldg(r0 + CH + 2));
  const float b01 = bf(__ldg(r1 + 2)), b11 = bf(__ldg(r1 + CH + 2));
  const float2 d10 = __ffma2_rn(a00, m1, a10), d01 = __ffma2_rn(a00, m1, a01);
  const float2 d11 = __ffma2_rn(d01, m1, __ffma2_rn(a10, m1, a11));
  float2 v = __fadd2_rn(a00, make_float2(-8388608.0f, -8388608.0f));
  v = __ffma2_rn(make_float2(fx, fx), d10, v);
  v = __ffma2_rn(make_float2(fy, fy), d01, v);
  v = __ffma2_rn(make_float2(fxy, fxy), d11, v);
  const float e10 = b10 - b00, e01 = b01 - b00, e11 = (b11 - b10) - e01;
  float vb = fmaf(fx, e10, b00 - 8388608.0f);
  vb = fmaf(fy, e01, vb);
  vb = fmaf(fxy, e11, vb);
  const float2 M = make_float2(12582912.0f, 12582912.0f);
  const float2 t = __fadd2_rn(v, M);
  const float2 dl = __ffma2_rn(__fadd2_rn(t, make_float2(-12582912.0f, -12582912.0f)), m1, v);
  const float tb = __fadd_rn(vb, 12582912.0f);
  const float db = __fsub_rn(vb, __fsub_rn(tb, 12582912.0f));
  ok = ok && fmaxf(fmaxf(fabsf(dl.x), fabsf(dl.y)), fabsf(db)) <= lim;
  const uint32_t rg = __byte_perm(__float_as_uint(t.x), __float_as_uint(t.y), 0x0040u);
  *out = __byte_perm(rg, __float_as_uint(tb), 0x0410u) | 0xFF000000u;
  return ok;
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
  int ixf, iyf;
  const float flx = floor_small(tx, &ixf), fly = floor_small(ty, &iyf);
  int x0 = a.ix + du + ixf;
  int y0 = a.iy + dv + iyf;
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
  float dmax = 0.0f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float d10 = v10[c] - v00[c], d01 = v01[c] - v00[c], d11 = (v11[c] - v10[c]) - d01;
    float v = fmaf(fx, d10, v00[c] - 8388608.0f);
    v = fmaf(fy, d01, v);
    v = fmaf(fxy, d11, v);
    float d;
    o[c] = round_near_u8(v, &d);
    dmax = fmaxf(dmax, d);
  }
  const bool tie = dmax > 0.5f - fmaxf(w.tie_band, kTieBand);
  if (tie) return sample_exact(w, s, X, Y);
  return pack_rgba(o[0], o[1], o[2], 255u);
}

}  // namespace fs
