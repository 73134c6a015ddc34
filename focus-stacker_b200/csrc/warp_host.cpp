// Host-side FP64 pose composition for libfocuscuda.
//
// Once per frame, the reference's per-pixel inverse transform
// (src/optimize.zig:3593-3635, src/remap.zig:377-441) is composed into a
// single projective map from output pixels to source pixels (plus the
// per-pixel radial inverse for lens poses).  All three reference paths are
// this map:
//   * basic rectilinear (yaw/pitch/roll/hfov): rectilinear(dest focal) ->
//     ray -> yaw -> pitch/roll -> rectilinear(image focal), which the
//     reference evaluates through the equirect/sphere chain
//     (src/optimize.zig:3618-3635);
//   * lens (radial and/or centre shift, no translation): the same rotation
//     with `world_to_local`, then the radial inverse (src/remap.zig:377-441);
//   * translation: plane hit minus the translation, W * (I - t n^T) applied
//     to the pano ray (the 1 / (n . ray) scale cancels in the projection,
//     src/optimize.zig:4009-4023, 3859-3881).
// The composition is checked against the reference's own chains by the
// tests (fs_inverse_map_points vs the oracle).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/focuscuda.h"
#include "fs_common.h"
#include "fs_host.h"

namespace fs {

namespace {

const double kPi = 3.14159265358979323846;

struct M3 {
  double m[3][3];
};

M3 mul(const M3& a, const M3& b) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) r.m[i][k] = a.m[i][0] * b.m[0][k] + a.m[i][1] * b.m[1][k] + a.m[i][2] * b.m[2][k];
  return r;
}
// Rotation conventions of the reference's setMatrix / yawMatrix
// (src/optimize.zig:3908-3944): world_to_local = Rz(roll) * Rx(-pitch) * Ry(-yaw).
M3 rot_x(double a) { return {{{1, 0, 0}, {0, std::cos(a), std::sin(a)}, {0, -std::sin(a), std::cos(a)}}}; }
M3 rot_y(double t) { return {{{std::cos(t), 0, -std::sin(t)}, {0, 1, 0}, {std::sin(t), 0, std::cos(t)}}}; }
M3 rot_z(double c) { return {{{std::cos(c), std::sin(c), 0}, {-std::sin(c), std::cos(c), 0}, {0, 0, 1}}}; }

double clampd(double v, double lo, double hi) { return std::max(lo, std::min(v, hi)); }
double focal_px(uint32_t width, double hfov_deg) {
  double h = clampd(hfov_deg, 1e-3, 179.0);
  return ((double)width * 0.5) / std::tan(h * kPi / 360.0);
}
bool has_translation(const fs_pose& p) {
  return std::fabs(p.trans_x) > 1e-12 || std::fabs(p.trans_y) > 1e-12 || std::fabs(p.trans_z) > 1e-12;
}
bool is_basic(const fs_pose& p) {
  return !has_translation(p) && std::fabs(p.radial_a) <= 1e-12 && std::fabs(p.radial_b) <= 1e-12 &&
         std::fabs(p.radial_c) <= 1e-12 && std::fabs(p.center_shift_x) <= 1e-12 &&
         std::fabs(p.center_shift_y) <= 1e-12;
}
bool has_radial_terms(const fs_pose& p) {  // exact-zero test of src/remap.zig:401
  return p.radial_a != 0.0 || p.radial_b != 0.0 || p.radial_c != 0.0;
}
double radial_inv_norm(uint32_t w, uint32_t h) {  // src/optimize.zig:4150-4156
  double hw = ((double)w - 1.0) * 0.5, hh = ((double)h - 1.0) * 0.5;
  double d = hw * hw + hh * hh;
  return d >= 1e-12 ? 1.0 / d : 1.0;
}

// Projective map (in homogeneous form) from ROI-relative output pixels to
// source pixels (centre included), and whether a radial inverse follows.
struct Composed {
  M3 H;            // (X, Y, 1) -> (Nx, Ny, Dn), source = (Nx/Dn, Ny/Dn) [radial space + centre for lens]
  bool radial;     // lens pose with non-zero radial terms
  bool basic;      // reference uses the basic-rectilinear chain
  double src_cx, src_cy, inv_norm;
};

Composed compose(const fs_pose& p, uint32_t w, uint32_t h, const fs_rect& roi) {
  Composed c;
  double dcx = ((double)w - 1.0) * 0.5, dcy = ((double)h - 1.0) * 0.5;  // panoramaCenter
  double df = focal_px(w, p.base_hfov_degrees);                          // dest focal
  double fi = focal_px(w, clampd(p.base_hfov_degrees + p.hfov_delta, 1e-3, 179.0));  // image focal
  c.src_cx = dcx;
  c.src_cy = dcy;
  c.inv_norm = radial_inv_norm(w, h);
  c.basic = is_basic(p);
  c.radial = !c.basic && has_radial_terms(p);
  // The basic chain rotates the +z-forward sphere vector by the transpose of
  // setMatrix(-pitch, 0, roll) after the yaw step (src/optimize.zig:3273-3291);
  // written in the -z-forward frame of the lens path that is
  // Rx(-pitch) Rz(-roll) Ry(-yaw): the roll turns the other way than in
  // world_to_local (src/optimize.zig:3575), and both are kept as they are.
  M3 W = c.basic ? mul(mul(rot_x(-p.pitch), rot_z(-p.roll)), rot_y(-p.yaw))
                 : mul(mul(rot_z(p.roll), rot_x(-p.pitch)), rot_y(-p.yaw));
  M3 T = {{{1, 0, (double)roi.left - dcx}, {0, 1, (double)roi.top - dcy}, {0, 0, -df}}};
  M3 A;
  if (has_translation(p)) {
    // plane normal = cartErect(tp_yaw, -tp_pitch, 1), src/optimize.zig:4045-4053, 3969-3971
    double phi = p.translation_plane_yaw, th = kPi * 0.5 + p.translation_plane_pitch;
    double n[3] = {std::sin(th) * std::sin(phi), std::cos(th), std::sin(th) * -std::cos(phi)};
    double t[3] = {p.trans_x, p.trans_y, p.trans_z};
    M3 P;
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) P.m[i][k] = (i == k ? 1.0 : 0.0) - t[i] * n[k];
    A = mul(mul(W, P), T);
  } else {
    A = mul(W, T);
  }
  double shx = c.basic ? 0.0 : p.center_shift_x, shy = c.basic ? 0.0 : p.center_shift_y;
  M3 K = {{{fi, 0, -(shx + dcx)}, {0, fi, -(shy + dcy)}, {0, 0, -1}}};
  c.H = mul(K, A);
  return c;
}

// Newton radial inverse with the reference's stopping rules (FP64),
// src/remap.zig:755-786.
void radial_inverse(const fs_pose& p, double inv_norm, double dx, double dy, double* ox, double* oy) {
  double q = std::sqrt(dx * dx + dy * dy);
  if (q < 1e-12) {
    *ox = dx;
    *oy = dy;
    return;
  }
  double r = q;
  for (int it = 0; it < 6; ++it) {
    double r2 = r * r * inv_norm, r4 = r2 * r2;
    double fac = 1.0 + p.radial_a * r2 + p.radial_b * r4 + p.radial_c * r4 * r2;
    double der = p.radial_a + 2.0 * p.radial_b * r2 + 3.0 * p.radial_c * r4;
    double f = r * fac - q;
    if (std::fabs(f) <= 1e-9) break;
    double dfd = fac + 2.0 * r * r * inv_norm * der;
    if (std::fabs(dfd) < 1e-12) break;
    r -= f / dfd;
    r = std::max(r, 0.0);
  }
  double s = r / q;
  *ox = dx * s;
  *oy = dy * s;
}

}  // namespace

static float fast_tie_band(const Warp& w, double ow, double oh);

bool compose_warp(const fs_pose& pose, uint32_t src_w, uint32_t src_h, const fs_rect& roi, Warp* out,
                  const char** why) {
  Composed c = compose(pose, src_w, src_h, roi);
  double h22 = c.H.m[2][2];
  if (!(std::fabs(h22) > 0.0) || !std::isfinite(h22)) {
    if (why) *why = "pose maps the output centre to infinity";
    return false;
  }
  double n[3][3];
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) n[i][k] = c.H.m[i][k] / h22;
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(n[i][k])) {
        if (why) *why = "non-finite pose";
        return false;
      }
  Warp w;
  std::memset(&w, 0, sizeof(w));
  w.kind = c.radial ? WARP_RADIAL : WARP_HOMOGRAPHY;
  w.a = n[0][0] - 1.0;
  w.b = n[0][1];
  w.c = n[0][2];
  w.d = n[1][0];
  w.e = n[1][1] - 1.0;
  w.f = n[1][2];
  w.g = n[2][0];
  w.h = n[2][1];
  w.src_cx = c.src_cx;
  w.src_cy = c.src_cy;
  w.radial_a = pose.radial_a;
  w.radial_b = pose.radial_b;
  w.radial_c = pose.radial_c;
  w.radial_inv_norm = c.inv_norm;
  // The denominator D = 1 + g X + h Y is affine: its extremes over the ROI
  // are at the corners.  The reference treats rays behind the camera as
  // empty samples (basic chain) or only rejects |denominator| < 1e-12 (lens
  // and translation paths); either way such pixels need the exact path.
  double ow = (double)(roi.right - roi.left), oh = (double)(roi.bottom - roi.top);
  double dmin = 1e300;
  for (int cy = 0; cy < 2; ++cy)
    for (int cx = 0; cx < 2; ++cx) {
      double X = cx ? ow : 0.0, Y = cy ? oh : 0.0;
      dmin = std::min(dmin, 1.0 + n[2][0] * X + n[2][1] * Y);
    }
  w.guard = dmin < 0.25 ? 1 : 0;
  w.tie_band = fast_tie_band(w, ow, oh);
  if (!(w.tie_band < 0.05f)) w.guard = 1;  // the fast sampler would decide too little: exact path only
  w.behind_is_void = c.basic ? 1 : 0;
  // the reference's |denominator| < 1e-12 is on -local_z; D is that scaled by 1/|h22|
  w.eps_den = 1e-12 / std::fabs(h22);
  *out = w;
  return true;
}

// Tie band of the device's fast FP32 sampler for this map.  Per 8x4 block
// the sampler takes the block anchor's FP64 position (fraction as two FP32
// words) and adds the offset of pixel (du, dv) from it, the FP32 rational
// (am1x du + bx dv - du (gam du + eta dv)) / (1 + gam du + eta dv) with
// coefficients rounded to FP32 (and likewise for y).  With T the sum of
// the absolute terms of that numerator, the position carries at most
// ~10 roundings of relative 2^-24 on T plus half an ulp of |position| <= 1 + T:
//   e_pos <= 2^-24 (1 + 11 T).
// The bilinear value moves by at most 255 per pixel of either coordinate
// and its own three FMAs round below 2^-16 each, so
//   e_val <= 510 e_pos + 6e-5,
// and twice that is the band.  T is largest at a corner of the ROI (the
// coefficients are ratios of affine functions of X and Y), evaluated there
// and at the centre with a 25% margin.
static float fast_tie_band(const Warp& w, double ow, double oh) {
  double T = 0.0;
  const double pts[5][2] = {{0, 0}, {ow, 0}, {0, oh}, {ow, oh}, {ow * 0.5, oh * 0.5}};
  for (const auto& pt : pts) {
    const double X = pt[0], Y = pt[1];
    const double D = 1.0 + w.g * X + w.h * Y;
    if (!(std::fabs(D) > 1e-3)) return 1.0f;
    const double dx = (w.a * X + w.b * Y + w.c - X * (w.g * X + w.h * Y)) / D;
    const double dy = (w.d * X + w.e * Y + w.f - Y * (w.g * X + w.h * Y)) / D;
    const double xa = X + dx, ya = Y + dy, dDa = D - 1.0;
    const double am1x = (w.a - xa * w.g - dDa) / D, bx = (w.b - xa * w.h) / D;
    const double ay = (w.d - ya * w.g) / D, bm1y = (w.e - ya * w.h - dDa) / D;
    const double gd = std::fabs(w.g / D) * 7.0 + std::fabs(w.h / D) * 3.0;
    T = std::max(T, std::fabs(am1x) * 7.0 + std::fabs(bx) * 3.0 + 7.0 * gd);
    T = std::max(T, std::fabs(ay) * 7.0 + std::fabs(bm1y) * 3.0 + 3.0 * gd);
  }
  T *= 1.25;
  const double e_pos = std::ldexp(1.0 + 11.0 * T, -24);
  const double band = 2.0 * (510.0 * e_pos + 6e-5);
  return (float)std::min(band, 1.0);
}

void inverse_map_point_f64(const fs_pose& pose, uint32_t w, uint32_t h, double x, double y, double* sx, double* sy) {
  fs_rect full = {0, 0, (int32_t)w, (int32_t)h};
  Composed c = compose(pose, w, h, full);
  double nx = c.H.m[0][0] * x + c.H.m[0][1] * y + c.H.m[0][2];
  double ny = c.H.m[1][0] * x + c.H.m[1][1] * y + c.H.m[1][2];
  double dn = c.H.m[2][0] * x + c.H.m[2][1] * y + c.H.m[2][2];
  double px = nx / dn, py = ny / dn;
  if (c.radial) {
    double ux, uy;
    radial_inverse(pose, c.inv_norm, px - c.src_cx, py - c.src_cy, &ux, &uy);
    px = c.src_cx + ux;
    py = c.src_cy + uy;
  }
  *sx = px;
  *sy = py;
}

// ------------------------------------------------------------------- ROI
// The common-overlap ROI (src/remap.zig:585-708) rounds polygon extremes
// with ceil/floor, so its result depends on the exact rounding residues of
// the reference's forward chain (an identity frame's corners come back
// +-1e-13 off the integer grid).  The forward map here therefore follows the
// reference's operation sequence (src/optimize.zig:3506-3525, 3659-3681,
// 3238-3364, 3784-3796, 3973-3982, 4071-4078) instead of the composed
// homography.
namespace {

struct P2 {
  double x, y;
};

P2 fwd_basic(const fs_pose& pose, double x, double y, uint32_t w, uint32_t h, bool* ok) {
  double cx = ((double)w - 1.0) * 0.5, cy = ((double)h - 1.0) * 0.5;
  double d = focal_px(w, pose.base_hfov_degrees);
  double fi = focal_px(w, clampd(pose.base_hfov_degrees + pose.hfov_delta, 1e-3, 179.0));
  double rs = d / fi;
  P2 p = {(x - cx) * rs, (y - cy) * rs};
  {  // rectilinear -> sphere (tangent-plane form)
    double r = std::sqrt(p.x * p.x + p.y * p.y) / d;
    double th = (r == 0.0) ? 1.0 : std::atan(r) / r;
    p = {th * p.x, th * p.y};
  }
  {  // rotate on the sphere by the pitch/roll matrix
    M3 m0 = mul(rot_z(pose.roll), rot_x(pose.pitch));
    M3 m = mul(m0, rot_y(0.0));
    double r = std::sqrt(p.x * p.x + p.y * p.y);
    double theta = r / d;
    double st = std::sin(theta);
    double rsc = (r == 0.0) ? 0.0 : st / r;
    double vx = rsc * p.x, vy = rsc * p.y, vz = std::cos(theta);
    double tx = m.m[0][0] * vx + m.m[1][0] * vy + m.m[2][0] * vz;
    double ty = m.m[0][1] * vx + m.m[1][1] * vy + m.m[2][1] * vz;
    double tz = m.m[0][2] * vx + m.m[1][2] * vy + m.m[2][2] * vz;
    double r2 = std::sqrt(tx * tx + ty * ty);
    double s = (r2 == 0.0) ? 0.0 : d * std::atan2(r2, tz) / r2;
    p = {s * tx, s * ty};
  }
  {  // sphere -> equirect
    double r = std::sqrt(p.x * p.x + p.y * p.y);
    double theta = r / d;
    double s = (theta == 0.0) ? 1.0 / d : std::sin(theta) / r;
    double v1 = s * p.x, v0 = std::cos(theta);
    p = {d * std::atan2(v1, v0), d * std::atan((s * p.y) / std::sqrt(v0 * v0 + v1 * v1))};
  }
  {  // yaw: shift the longitude, wrapping at +-180 degrees
    double half = d * kPi, turn = pose.yaw * d;
    double xx = p.x + turn, full = 2.0 * half;
    if (xx < -half) {
      xx += full;
      while (xx < -half) xx += full;
    } else if (xx > half) {
      xx -= full;
      while (xx > half) xx -= full;
    }
    p.x = xx;
  }
  double phi = p.x / d;
  if (phi < -kPi * 0.5 || phi > kPi * 0.5) {
    *ok = false;
    return {-1.0, -1.0};
  }
  double theta = -(p.y / d) + kPi * 0.5;
  *ok = true;
  return {cx + d * std::tan(phi), cy + d / (std::tan(theta) * std::cos(phi))};
}

P2 fwd_point(const fs_pose& pose, double x, double y, uint32_t w, uint32_t h) {
  bool ok = true;
  if (is_basic(pose)) return fwd_basic(pose, x, y, w, h, &ok);
  double cx = ((double)w - 1.0) * 0.5, cy = ((double)h - 1.0) * 0.5;
  double d = focal_px(w, pose.base_hfov_degrees);
  double sx = (x - cx) - pose.center_shift_x, sy = (y - cy) - pose.center_shift_y;
  double r2 = (sx * sx + sy * sy) * radial_inv_norm(w, h);
  double r4 = r2 * r2, r6 = r4 * r2;
  double fac = 1.0 + pose.radial_a * r2 + pose.radial_b * r4 + pose.radial_c * r6;
  double dx = sx * fac, dy = sy * fac;
  double fs_ = focal_px(w, clampd(pose.base_hfov_degrees + pose.hfov_delta, 1e-3, 179.0));
  double lx = dx, ly = dy, lz = -fs_;
  double nrm = std::sqrt(lx * lx + ly * ly + lz * lz);
  if (nrm < 1e-12) {
    lx = 0; ly = 0; lz = 1;
  } else {
    lx /= nrm; ly /= nrm; lz /= nrm;
  }
  M3 m = mul(mul(rot_z(pose.roll), rot_x(-pose.pitch)), rot_y(0.0));
  double ix = m.m[0][0] * lx + m.m[1][0] * ly + m.m[2][0] * lz;
  double iy = m.m[0][1] * lx + m.m[1][1] * ly + m.m[2][1] * lz;
  double iz = m.m[0][2] * lx + m.m[1][2] * ly + m.m[2][2] * lz;
  double c = std::cos(pose.yaw), s = std::sin(pose.yaw);
  double rx = c * ix - s * iz, ry = iy, rz = s * ix + c * iz;
  if (has_translation(pose)) {
    double phi = pose.translation_plane_yaw, th = kPi * 0.5 - (-pose.translation_plane_pitch / 1.0);
    double n[3] = {std::sin(th) * std::sin(phi), std::cos(th), std::sin(th) * -std::cos(phi)};
    double cam[3] = {pose.trans_x, pose.trans_y, pose.trans_z};
    double tgt[3] = {cam[0] + rx, cam[1] + ry, cam[2] + rz};
    double dir[3] = {tgt[0] - cam[0], tgt[1] - cam[1], tgt[2] - cam[2]};
    double num = 1.0 - (n[0] * cam[0] + n[1] * cam[1] + n[2] * cam[2]);
    double den = n[0] * dir[0] + n[1] * dir[1] + n[2] * dir[2];
    if (std::fabs(den) < 1e-12) {
      rx = 0; ry = 0; rz = 1;
    } else {
      double u = num / den;
      rx = cam[0] + u * dir[0];
      ry = cam[1] + u * dir[1];
      rz = cam[2] + u * dir[2];
    }
  }
  double den = -rz;
  if (den <= 1e-12) return {-1.0, -1.0};
  return {cx + d * (rx / den), cy + d * (ry / den)};
}

bool inside_edge(P2 p, P2 a, P2 b) { return ((b.x - a.x) * (p.y - a.y) - (b.y - a.y) * (p.x - a.x)) >= -1e-6; }
P2 intersect(P2 p1, P2 p2, P2 q1, P2 q2) {
  double a1 = p2.y - p1.y, b1 = p1.x - p2.x, c1 = a1 * p1.x + b1 * p1.y;
  double a2 = q2.y - q1.y, b2 = q1.x - q2.x, c2 = a2 * q1.x + b2 * q1.y;
  double det = a1 * b2 - a2 * b1;
  if (std::fabs(det) < 1e-9) return p2;
  return {(b2 * c1 - b1 * c2) / det, (a1 * c2 - a2 * c1) / det};
}
std::vector<P2> clip(const std::vector<P2>& subject, const std::vector<P2>& clipper) {
  std::vector<P2> cur = subject;
  for (size_t i = 0; i < clipper.size() && !cur.empty(); ++i) {
    P2 a = clipper[i], b = clipper[(i + 1) % clipper.size()];
    std::vector<P2> next;
    P2 prev = cur.back();
    bool pin = inside_edge(prev, a, b);
    for (const P2& q : cur) {
      bool qin = inside_edge(q, a, b);
      if (qin != pin) next.push_back(intersect(prev, q, a, b));
      if (qin) next.push_back(q);
      prev = q;
      pin = qin;
    }
    cur.swap(next);
  }
  return cur;
}

}  // namespace

void forward_map_point(const fs_pose& pose, uint32_t w, uint32_t h, double x, double y, double* ox, double* oy) {
  P2 p = fwd_point(pose, x, y, w, h);
  *ox = p.x;
  *oy = p.y;
}

bool compute_roi(const fs_pose* poses, const uint32_t* widths, const uint32_t* heights, const uint8_t* active,
                 size_t n, fs_rect* out) {
  std::vector<P2> poly;
  bool first = true;
  for (size_t i = 0; i < n; ++i) {
    if (active && !active[i]) continue;
    uint32_t w = widths[i], h = heights[i];
    std::vector<P2> quad = {fwd_point(poses[i], 0, 0, w, h), fwd_point(poses[i], (double)(w - 1), 0, w, h),
                            fwd_point(poses[i], (double)(w - 1), (double)(h - 1), w, h),
                            fwd_point(poses[i], 0, (double)(h - 1), w, h)};
    if (first) {
      poly = quad;
      first = false;
    } else {
      poly = clip(poly, quad);
      if (poly.empty()) return false;
    }
  }
  if (poly.empty()) return false;
  double x0 = poly[0].x, x1 = poly[0].x, y0 = poly[0].y, y1 = poly[0].y;
  for (const P2& q : poly) {
    x0 = std::min(x0, q.x);
    x1 = std::max(x1, q.x);
    y0 = std::min(y0, q.y);
    y1 = std::max(y1, q.y);
  }
  fs_rect r = {(int32_t)std::ceil(x0), (int32_t)std::ceil(y0), (int32_t)std::floor(x1) + 1, (int32_t)std::floor(y1) + 1};
  if (r.right <= r.left || r.bottom <= r.top) return false;
  *out = r;
  return true;
}

}  // namespace fs
