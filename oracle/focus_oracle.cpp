// CPU oracle for the remap + pyramid-contrast fusion path.
//
// TEST INFRASTRUCTURE ONLY.  This file is a line-by-line C++ restatement of
// the reference (asingleoat/focus-stacker, Zig) functions on the hot path.  It
// is used by tests/, by __graft_entry__.smoke() and by bench.py's
// cpu_baseline / --impl reference legs as the checker and the timed CPU
// baseline.  Nothing in the shipped library links or calls it.
//
// The reference itself (Zig 0.15 + libjpeg/libpng/libtiff/libexif) cannot be
// built in this image (no `zig`, no image libraries), so this restatement is
// the oracle.  It is pinned against every known-answer test the reference
// holds for this path (tests/test_oracle_kat.py) and against the reference's
// own identity-remap golden TIFF (tests/golden/).
//
// Semantics kept from the Zig source:
//   * strict IEEE arithmetic, no FMA contraction (built with
//     -ffp-contract=off -fno-fast-math);
//   * @round = round half away from zero (C `round`), @intFromFloat truncates;
//   * f64 in the pose maths, the remap and the contrast sums; f32 elsewhere
//     (Real = float).  Real = double gives the FP64 evaluation of the same
//     pyramid used to measure precision forms.
//
// Every function cites the reference file:line it follows (paths relative to
// the reference project root).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------- pose maths
// src/optimize.zig:32-48 (ImagePose); field order matches the C-ABI fs_pose.
struct ImagePose {
  double yaw = 0, pitch = 0, roll = 0, hfov_delta = 0;
  double trans_x = 0, trans_y = 0, trans_z = 0;
  double translation_plane_yaw = 0, translation_plane_pitch = 0;
  double radial_a = 0, radial_b = 0, radial_c = 0;
  double center_shift_x = 0, center_shift_y = 0;
  double base_hfov_degrees = 50.0;
};

struct Point2 { double x, y; };
struct Vec3 { double x, y, z; };
typedef double Matrix3[3][3];

static const double kPi = 3.14159265358979323846;

static double clampd(double v, double lo, double hi) {  // std.math.clamp
  return std::max(lo, std::min(v, hi));
}

// src/optimize.zig:3074-3081
static bool hasTranslation(const ImagePose& p) {  // src/optimize.zig:3965-3967
  return std::fabs(p.trans_x) > 1e-12 || std::fabs(p.trans_y) > 1e-12 || std::fabs(p.trans_z) > 1e-12;
}
static bool hasBasicRectilinearPose(const ImagePose& p) {
  return !hasTranslation(p) && std::fabs(p.radial_a) <= 1e-12 && std::fabs(p.radial_b) <= 1e-12 &&
         std::fabs(p.radial_c) <= 1e-12 && std::fabs(p.center_shift_x) <= 1e-12 &&
         std::fabs(p.center_shift_y) <= 1e-12;
}

// src/optimize.zig:3705-3723
static double focalLengthPixels(uint32_t width, double hfov_degrees) {
  double clamped = clampd(hfov_degrees, 1e-3, 179.0);
  return ((double)width * 0.5) / std::tan(clamped * kPi / 360.0);
}
static Point2 panoramaCenter(uint32_t w, uint32_t h) {
  return {((double)w - 1.0) * 0.5, ((double)h - 1.0) * 0.5};
}
static double panoramaFocalLengthPixels(uint32_t w, const ImagePose& p) {
  return focalLengthPixels(w, p.base_hfov_degrees);
}
static double effectiveHfovDegrees(const ImagePose& p) {
  return clampd(p.base_hfov_degrees + p.hfov_delta, 1e-3, 179.0);
}
// src/optimize.zig:4080-4086
static Point2 distortionCenter(uint32_t w, uint32_t h) { return panoramaCenter(w, h); }

// src/optimize.zig:3730-3738
static Vec3 normalize3(Vec3 v) {
  double norm = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
  if (norm < 1e-12) return {0, 0, 1};
  return {v.x / norm, v.y / norm, v.z / norm};
}

// src/optimize.zig:3908-3963
static void setMatrix(double a, double b, double c, bool cl, Matrix3 out);
static void matrixMatrixMul(const Matrix3 m1, const Matrix3 m2, Matrix3 out) {
  Matrix3 r;
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) r[i][k] = m1[i][0] * m2[0][k] + m1[i][1] * m2[1][k] + m1[i][2] * m2[2][k];
  std::memcpy(out, r, sizeof(r));
}
static void setMatrix(double a, double b, double c, bool cl, Matrix3 out) {
  Matrix3 mx = {{1.0, 0.0, 0.0}, {0.0, std::cos(a), std::sin(a)}, {0.0, -std::sin(a), std::cos(a)}};
  Matrix3 my = {{std::cos(b), 0.0, -std::sin(b)}, {0.0, 1.0, 0.0}, {std::sin(b), 0.0, std::cos(b)}};
  Matrix3 mz = {{std::cos(c), std::sin(c), 0.0}, {-std::sin(c), std::cos(c), 0.0}, {0.0, 0.0, 1.0}};
  Matrix3 dummy;
  if (cl) matrixMatrixMul(mz, mx, dummy); else matrixMatrixMul(mx, mz, dummy);
  matrixMatrixMul(dummy, my, out);
}
static void yawMatrix(double yaw, Matrix3 out) {
  double c = std::cos(yaw), s = std::sin(yaw);
  Matrix3 m = {{c, 0.0, -s}, {0.0, 1.0, 0.0}, {s, 0.0, c}};
  std::memcpy(out, m, sizeof(m));
}
static Vec3 matrixMul(const Matrix3 m, Vec3 v) {
  return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
          m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
}
static Vec3 matrixInvMul(const Matrix3 m, Vec3 v) {
  return {m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
          m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z};
}
// src/optimize.zig:3896-3905
static Vec3 rotateYaw(Vec3 r, double yaw) {
  double c = std::cos(yaw), s = std::sin(yaw);
  return {c * r.x - s * r.z, r.y, s * r.x + c * r.z};
}
// src/optimize.zig:4045-4053
static Vec3 cartErect(double x, double y, double distance) {
  double phi = x / distance;
  double theta_zenith = kPi * 0.5 - (y / distance);
  return {std::sin(theta_zenith) * std::sin(phi), std::cos(theta_zenith), std::sin(theta_zenith) * -std::cos(phi)};
}
static double dot3(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// src/optimize.zig:3969-3971
static Vec3 translationPlaneNormal(const ImagePose& p) {
  return cartErect(p.translation_plane_yaw, -p.translation_plane_pitch, 1.0);
}
// src/optimize.zig:4025-4043
static bool linePlaneIntersection(Vec3 normal, Vec3 p1, Vec3 p2, Vec3* out) {
  Vec3 d = {p2.x - p1.x, p2.y - p1.y, p2.z - p1.z};
  double numerator = 1.0 - dot3(normal, p1);
  double denominator = dot3(normal, d);
  if (std::fabs(denominator) < 1e-12) return false;
  double u = numerator / denominator;
  *out = {p1.x + u * d.x, p1.y + u * d.y, p1.z + u * d.z};
  return true;
}
// src/optimize.zig:4150-4156
static double radialNormalizer(uint32_t w, uint32_t h) {
  double hw = ((double)w - 1.0) * 0.5, hh = ((double)h - 1.0) * 0.5;
  double denom = hw * hw + hh * hh;
  if (denom >= 1e-12) return 1.0 / denom;
  return 1.0;
}

// src/optimize.zig:3527-3586
struct InverseTransformCache {
  bool basic_rectilinear, has_translation;
  double src_center_x, src_center_y, dest_center_x, dest_center_y;
  double pano_distance, half_turn, resize_scale, dest_focal, image_focal;
  Matrix3 pitch_roll, world_to_local;
  double yaw_turn, yaw;
  double radial_a, radial_b, radial_c, center_shift_x, center_shift_y, radial_inv_norm;
  double trans_x, trans_y, trans_z;
  Vec3 translation_plane_normal;
};

static InverseTransformCache initInverseTransformCache(const ImagePose& pose, uint32_t width, uint32_t height) {
  InverseTransformCache c;
  Point2 sc = distortionCenter(width, height);
  Point2 dc = panoramaCenter(width, height);
  double pano_distance = panoramaFocalLengthPixels(width, pose);
  c.basic_rectilinear = hasBasicRectilinearPose(pose);
  c.has_translation = hasTranslation(pose);
  c.src_center_x = sc.x; c.src_center_y = sc.y;
  c.dest_center_x = dc.x; c.dest_center_y = dc.y;
  c.pano_distance = pano_distance;
  c.half_turn = pano_distance * kPi;
  c.resize_scale = focalLengthPixels(width, effectiveHfovDegrees(pose)) / pano_distance;
  c.dest_focal = pano_distance;
  c.image_focal = focalLengthPixels(width, effectiveHfovDegrees(pose));
  setMatrix(-pose.pitch, 0.0, pose.roll, true, c.pitch_roll);
  Matrix3 pr, ym;
  setMatrix(-pose.pitch, 0.0, pose.roll, true, pr);
  yawMatrix(-pose.yaw, ym);
  matrixMatrixMul(pr, ym, c.world_to_local);
  c.yaw_turn = -pose.yaw * pano_distance;
  c.yaw = pose.yaw;
  c.radial_a = pose.radial_a; c.radial_b = pose.radial_b; c.radial_c = pose.radial_c;
  c.center_shift_x = pose.center_shift_x; c.center_shift_y = pose.center_shift_y;
  c.radial_inv_norm = radialNormalizer(width, height);
  c.trans_x = pose.trans_x; c.trans_y = pose.trans_y; c.trans_z = pose.trans_z;
  c.translation_plane_normal = translationPlaneNormal(pose);
  return c;
}

// src/optimize.zig:3340-3364, 3247-3271, 3273-3291, 3309-3323 (legacy chain pieces)
static Point2 erectRectPoint(Point2 p, double d) {
  return {d * std::atan2(p.x, d), d * std::atan2(p.y, std::sqrt(d * d + p.x * p.x))};
}
static Point2 rotateErectPoint(Point2 p, double half_turn, double turn) {
  double x = p.x + turn;
  double full = 2.0 * half_turn;
  if (x < -half_turn) {
    x += full;
    while (x < -half_turn) x += full;
  } else if (x > half_turn) {
    x -= full;
    while (x > half_turn) x -= full;
  }
  return {x, p.y};
}
static Point2 sphereTpErectPoint(Point2 p, double d) {
  double phi = p.x / d;
  double theta = -(p.y / d) + kPi * 0.5;
  if (theta < 0.0) { theta = -theta; phi += kPi; }
  if (theta > kPi) { theta = kPi - (theta - kPi); phi += kPi; }
  double s = std::sin(theta);
  double v0 = s * std::sin(phi);
  double v1 = std::cos(theta);
  double r = std::sqrt(v1 * v1 + v0 * v0);
  double scale = (r == 0.0) ? 0.0 : d * std::atan2(r, s * std::cos(phi)) / r;
  return {scale * v0, scale * v1};
}
static Point2 perspSpherePoint(Point2 p, const Matrix3 m, double d) {
  double px = p.x, py = p.y;
  double r = std::sqrt(px * px + py * py);
  double theta = r / d;
  double sin_theta = std::sin(theta);
  double radial_scale = (r == 0.0) ? 0.0 : sin_theta / r;
  double vx = radial_scale * px, vy = radial_scale * py, vz = std::cos(theta);
  double tx = m[0][0] * vx + m[1][0] * vy + m[2][0] * vz;
  double ty = m[0][1] * vx + m[1][1] * vy + m[2][1] * vz;
  double tz = m[0][2] * vx + m[1][2] * vy + m[2][2] * vz;
  double r2 = std::sqrt(tx * tx + ty * ty);
  double scale = (r2 == 0.0) ? 0.0 : d * std::atan2(r2, tz) / r2;
  return {scale * tx, scale * ty};
}
static Point2 rectSphereTpPoint(Point2 p, double d) {
  double r = std::sqrt(p.x * p.x + p.y * p.y);
  double theta = r / d;
  double rho = (theta >= kPi * 0.5) ? 1.6e16 : (theta == 0.0 ? 1.0 : std::tan(theta) / theta);
  return {rho * p.x, rho * p.y};
}
// forward-chain pieces, src/optimize.zig:3238-3245, 3293-3307, 3325-3338
static Point2 sphereTpRectPoint(Point2 p, double d) {
  double r = std::sqrt(p.x * p.x + p.y * p.y) / d;
  double theta = (r == 0.0) ? 1.0 : std::atan(r) / r;
  return {theta * p.x, theta * p.y};
}
static Point2 erectSphereTpPoint(Point2 p, double d) {
  double r = std::sqrt(p.x * p.x + p.y * p.y);
  double theta = r / d;
  double s = (theta == 0.0) ? 1.0 / d : std::sin(theta) / r;
  double v1 = s * p.x;
  double v0 = std::cos(theta);
  return {d * std::atan2(v1, v0), d * std::atan((s * p.y) / std::sqrt(v0 * v0 + v1 * v1))};
}
static bool rectErectPoint(Point2 p, double d, Point2* out) {
  double phi = p.x / d;
  if (phi < -kPi * 0.5 || phi > kPi * 0.5) return false;
  double theta = -(p.y / d) + kPi * 0.5;
  *out = {d * std::tan(phi), d / (std::tan(theta) * std::cos(phi))};
  return true;
}

// src/optimize.zig:3618-3635
static Point2 basicRectilinearInverseTransformPointCachedLegacy(const InverseTransformCache& c, double ox, double oy) {
  Point2 p = {ox - c.dest_center_x, oy - c.dest_center_y};
  p = erectRectPoint(p, c.pano_distance);
  p = rotateErectPoint(p, c.half_turn, c.yaw_turn);
  p = sphereTpErectPoint(p, c.pano_distance);
  p = perspSpherePoint(p, c.pitch_roll, c.pano_distance);
  p = rectSphereTpPoint(p, c.pano_distance);
  p.x *= c.resize_scale;
  p.y *= c.resize_scale;
  return {c.src_center_x + p.x, c.src_center_y + p.y};
}

// src/optimize.zig:4009-4023
static bool rayFromTranslationPlaneCachedUnnormalized(const InverseTransformCache& c, Vec3 pano_ray, Vec3* out) {
  Vec3 hit;
  if (!linePlaneIntersection(c.translation_plane_normal, {0, 0, 0}, pano_ray, &hit)) return false;
  *out = {hit.x - c.trans_x, hit.y - c.trans_y, hit.z - c.trans_z};
  return true;
}
// src/optimize.zig:3859-3881
static Point2 imagePlaneFromWorldRayCached(const InverseTransformCache& c, Vec3 w) {
  double lx = c.world_to_local[0][0] * w.x + c.world_to_local[0][1] * w.y + c.world_to_local[0][2] * w.z;
  double ly = c.world_to_local[1][0] * w.x + c.world_to_local[1][1] * w.y + c.world_to_local[1][2] * w.z;
  double lz = c.world_to_local[2][0] * w.x + c.world_to_local[2][1] * w.y + c.world_to_local[2][2] * w.z;
  double denom = -lz;
  if (std::fabs(denom) < 1e-12) return {-1.0, -1.0};
  return {c.image_focal * (lx / denom) + c.center_shift_x, c.image_focal * (ly / denom) + c.center_shift_y};
}
// src/optimize.zig:4204-4235
static Point2 invertRadialDistortionCached(const InverseTransformCache& c, double dx, double dy) {
  double q_radius = std::sqrt(dx * dx + dy * dy);
  if (q_radius < 1e-12) return {dx, dy};
  double radius = q_radius;
  for (int it = 0; it < 6; ++it) {
    double r2 = radius * radius * c.radial_inv_norm;
    double r4 = r2 * r2;
    double factor = 1.0 + c.radial_a * r2 + c.radial_b * r4 + c.radial_c * r4 * r2;
    double fd = c.radial_a + 2.0 * c.radial_b * r2 + 3.0 * c.radial_c * r4;
    double f = radius * factor - q_radius;
    if (std::fabs(f) <= 1e-9) break;
    double df = factor + 2.0 * radius * radius * c.radial_inv_norm * fd;
    if (std::fabs(df) < 1e-12) break;
    radius -= f / df;
    radius = std::max(radius, 0.0);
  }
  double scale = radius / q_radius;
  return {dx * scale, dy * scale};
}
// src/optimize.zig:3593-3616
static Point2 inverseTransformPointCached(const InverseTransformCache& c, double ox, double oy) {
  if (c.basic_rectilinear) return basicRectilinearInverseTransformPointCachedLegacy(c, ox, oy);
  Vec3 pano_ray = {ox - c.dest_center_x, oy - c.dest_center_y, -c.dest_focal};
  Vec3 camera_ray = pano_ray;
  if (c.has_translation) {
    if (!rayFromTranslationPlaneCachedUnnormalized(c, pano_ray, &camera_ray)) return {-1.0, -1.0};
  }
  Point2 radial = imagePlaneFromWorldRayCached(c, camera_ray);
  Point2 u = invertRadialDistortionCached(c, radial.x, radial.y);
  return {c.src_center_x + u.x, c.src_center_y + u.y};
}
// src/remap.zig:755-786
static Point2 undistortSourcePoint(const InverseTransformCache& c, double dx, double dy) {
  double q_radius = std::sqrt(dx * dx + dy * dy);
  if (q_radius < 1e-12) return {c.src_center_x + dx, c.src_center_y + dy};
  double radius = q_radius;
  for (int it = 0; it < 6; ++it) {
    double r2 = radius * radius * c.radial_inv_norm;
    double r4 = r2 * r2;
    double factor = 1.0 + c.radial_a * r2 + c.radial_b * r4 + c.radial_c * r4 * r2;
    double fd = c.radial_a + 2.0 * c.radial_b * r2 + 3.0 * c.radial_c * r4;
    double f = radius * factor - q_radius;
    if (std::fabs(f) <= 1e-9) break;
    double df = factor + 2.0 * radius * radius * c.radial_inv_norm * fd;
    if (std::fabs(df) < 1e-12) break;
    radius -= f / df;
    radius = std::max(radius, 0.0);
  }
  double scale = radius / q_radius;
  return {c.src_center_x + (dx * scale), c.src_center_y + (dy * scale)};
}

// forward map, src/optimize.zig:3506-3525 and 3659-3681, 3784-3796, 3973-3982, 4071-4078, 4158-4171
static double radialScale(const ImagePose& p, double r2) {
  double r4 = r2 * r2, r6 = r4 * r2;
  return 1.0 + p.radial_a * r2 + p.radial_b * r4 + p.radial_c * r6;
}
static Point2 basicRectilinearTransformPoint(const ImagePose& pose, double x, double y, uint32_t w, uint32_t h) {
  Point2 sc = distortionCenter(w, h), dc = panoramaCenter(w, h);
  double pano_distance = panoramaFocalLengthPixels(w, pose);
  double image_focal = focalLengthPixels(w, effectiveHfovDegrees(pose));
  double resize_scale = pano_distance / image_focal;
  Point2 p = {(x - sc.x) * resize_scale, (y - sc.y) * resize_scale};
  p = sphereTpRectPoint(p, pano_distance);
  Matrix3 m;
  setMatrix(pose.pitch, 0.0, pose.roll, true, m);
  p = perspSpherePoint(p, m, pano_distance);
  p = erectSphereTpPoint(p, pano_distance);
  p = rotateErectPoint(p, pano_distance * kPi, pose.yaw * pano_distance);
  Point2 q;
  if (!rectErectPoint(p, pano_distance, &q)) return {-1.0, -1.0};
  return {dc.x + q.x, dc.y + q.y};
}
static Point2 transformPoint(const ImagePose& pose, double xf, double yf, uint32_t w, uint32_t h) {
  if (hasBasicRectilinearPose(pose)) return basicRectilinearTransformPoint(pose, xf, yf, w, h);
  Point2 sc = distortionCenter(w, h), dc = panoramaCenter(w, h);
  double dest_focal = panoramaFocalLengthPixels(w, pose);
  // sourceWorldRay, src/optimize.zig:3784-3796
  double sx = (xf - sc.x) - pose.center_shift_x, sy = (yf - sc.y) - pose.center_shift_y;
  double r2 = (sx * sx + sy * sy) * radialNormalizer(w, h);
  double factor = radialScale(pose, r2);
  double distx = sx * factor, disty = sy * factor;
  double src_focal = focalLengthPixels(w, effectiveHfovDegrees(pose));
  Vec3 local = normalize3({distx, disty, -src_focal});
  Matrix3 pr;
  setMatrix(-pose.pitch, 0.0, pose.roll, true, pr);
  Vec3 ray = rotateYaw(matrixInvMul(pr, local), pose.yaw);
  Vec3 projected = ray;
  if (hasTranslation(pose)) {  // projectViaTranslationPlane, src/optimize.zig:3973-3982
    Vec3 camera = {pose.trans_x, pose.trans_y, pose.trans_z};
    Vec3 target = {camera.x + ray.x, camera.y + ray.y, camera.z + ray.z};
    if (!linePlaneIntersection(translationPlaneNormal(pose), camera, target, &projected)) projected = {0.0, 0.0, 1.0};
  }
  double denom = -projected.z;  // projectRectilinear, src/optimize.zig:4071-4078
  if (denom <= 1e-12) return {-1.0, -1.0};
  return {dc.x + dest_focal * (projected.x / denom), dc.y + dest_focal * (projected.y / denom)};
}

// -------------------------------------------------------------------- remap
struct Rect { int32_t left, top, right, bottom; };

static inline bool inBounds(int32_t x, int32_t y, uint32_t w, uint32_t h) {  // src/remap.zig:996-998
  return x >= 0 && y >= 0 && x < (int32_t)w && y < (int32_t)h;
}

// src/remap.zig:710-753 (u8) and 841-884 (u16), with the interior
// (src/remap.zig:788-839) and soft-edge (src/remap.zig:939-994) helpers.
template <typename T>
static void samplePixelBilinear(T* dst, const T* pixels, uint32_t width, uint32_t height, int src_channels,
                                int dst_channels, double x, double y, double maxv) {
  int32_t x0 = (int32_t)std::floor(x), y0 = (int32_t)std::floor(y);
  int32_t x1 = x0 + 1, y1 = y0 + 1;
  double fx = x - (double)x0, fy = y - (double)y0;
  double omfx = 1.0 - fx, omfy = 1.0 - fy;
  double w00 = omfx * omfy, w10 = fx * omfy, w01 = omfx * fy, w11 = fx * fy;
  if (x0 >= 0 && y0 >= 0 && x1 < (int32_t)width && y1 < (int32_t)height) {
    size_t row_stride = (size_t)width * src_channels;
    size_t b00 = (size_t)y0 * row_stride + (size_t)x0 * src_channels;
    size_t b10 = b00 + src_channels, b01 = b00 + row_stride, b11 = b01 + src_channels;
    double support = w00 + w10 + w01 + w11;
    for (int ch = 0; ch < src_channels; ++ch) {
      double value = (double)pixels[b00 + ch] * w00 + (double)pixels[b10 + ch] * w10 + (double)pixels[b01 + ch] * w01 +
                     (double)pixels[b11 + ch] * w11;
      dst[ch] = (T)std::round(value / support);
    }
    if (dst_channels > src_channels) dst[src_channels] = (T)maxv;
    return;
  }
  double support = 0.0;
  if (inBounds(x0, y0, width, height)) support += w00;
  if (inBounds(x1, y0, width, height)) support += w10;
  if (inBounds(x0, y1, width, height)) support += w01;
  if (inBounds(x1, y1, width, height)) support += w11;
  if (support <= 0.0) {
    for (int ch = 0; ch < dst_channels; ++ch) dst[ch] = 0;
    return;
  }
  for (int ch = 0; ch < src_channels; ++ch) {
    double value = 0.0;
    auto at = [&](int32_t xx, int32_t yy) {
      return (double)pixels[((size_t)yy * width + (size_t)xx) * src_channels + ch];
    };
    if (inBounds(x0, y0, width, height)) value += at(x0, y0) * w00;
    if (inBounds(x1, y0, width, height)) value += at(x1, y0) * w10;
    if (inBounds(x0, y1, width, height)) value += at(x0, y1) * w01;
    if (inBounds(x1, y1, width, height)) value += at(x1, y1) * w11;
    dst[ch] = (T)std::round(value / support);
  }
  if (dst_channels > src_channels) dst[src_channels] = (T)std::round(support * maxv);
}

// src/remap.zig:343-441 (u8) and 443-541 (u16)
template <typename T>
static void remapRows(T* dst, const T* src, uint32_t width, uint32_t height, int src_channels, int dst_channels,
                      Rect roi, const InverseTransformCache& cache, uint32_t out_width, uint32_t row_start,
                      uint32_t row_end, double maxv) {
  if (!cache.basic_rectilinear && !cache.has_translation) {
    // remapU8RowsNoTranslationLens, src/remap.zig:377-441
    double roi_left = (double)roi.left, roi_top = (double)roi.top;
    double sx_x = cache.world_to_local[0][0], sx_y = cache.world_to_local[1][0], sx_z = cache.world_to_local[2][0];
    double constant_z = -cache.dest_focal;
    double base_x = roi_left - cache.dest_center_x;
    bool radial = cache.radial_a != 0.0 || cache.radial_b != 0.0 || cache.radial_c != 0.0;
    for (uint32_t y = row_start; y < row_end; ++y) {
      double pano_y = (roi_top + (double)y) - cache.dest_center_y;
      double lx = cache.world_to_local[0][0] * base_x + cache.world_to_local[0][1] * pano_y +
                  cache.world_to_local[0][2] * constant_z;
      double ly = cache.world_to_local[1][0] * base_x + cache.world_to_local[1][1] * pano_y +
                  cache.world_to_local[1][2] * constant_z;
      double lz = cache.world_to_local[2][0] * base_x + cache.world_to_local[2][1] * pano_y +
                  cache.world_to_local[2][2] * constant_z;
      size_t dst_base = ((size_t)y * out_width) * dst_channels;
      for (uint32_t i = 0; i < out_width; ++i) {
        double denom = -lz;
        if (std::fabs(denom) < 1e-12) {
          for (int ch = 0; ch < dst_channels; ++ch) dst[dst_base + ch] = 0;
        } else {
          double rx = cache.image_focal * (lx / denom) + cache.center_shift_x;
          double ry = cache.image_focal * (ly / denom) + cache.center_shift_y;
          Point2 s = radial ? undistortSourcePoint(cache, rx, ry)
                            : Point2{cache.src_center_x + rx, cache.src_center_y + ry};
          samplePixelBilinear<T>(dst + dst_base, src, width, height, src_channels, dst_channels, s.x, s.y, maxv);
        }
        dst_base += dst_channels;
        lx += sx_x;
        ly += sx_y;
        lz += sx_z;
      }
    }
    return;
  }
  double roi_left = (double)roi.left, roi_top = (double)roi.top;
  for (uint32_t y = row_start; y < row_end; ++y) {
    double world_y = roi_top + (double)y;
    double world_x = roi_left;
    size_t dst_base = ((size_t)y * out_width) * dst_channels;
    for (uint32_t i = 0; i < out_width; ++i) {
      Point2 s = inverseTransformPointCached(cache, world_x, world_y);
      samplePixelBilinear<T>(dst + dst_base, src, width, height, src_channels, dst_channels, s.x, s.y, maxv);
      dst_base += dst_channels;
      world_x += 1.0;
    }
  }
}

// Fork-join over row ranges with the reference's partition
// (rows_per_worker = ceil(rows / workers); worker i gets [i*rpw, (i+1)*rpw)),
// e.g. src/remap.zig:240-277, src/fuse/pyramid.zig:653-684.
template <typename F>
static void parallelRows(uint32_t rows, int jobs, F&& fn) {
  int workers = std::max(1, std::min(jobs, (int)rows));
  if (workers <= 1) {
    fn(0u, rows);
    return;
  }
  uint32_t rpw = (rows + workers - 1) / workers;
  std::vector<std::thread> threads;
  for (int i = 1; i < workers; ++i) {
    uint32_t s = std::min<uint32_t>(i * rpw, rows), e = std::min<uint32_t>(s + rpw, rows);
    threads.emplace_back([&fn, s, e] { if (s < e) fn(s, e); });
  }
  fn(0u, std::min(rpw, rows));
  for (auto& t : threads) t.join();
}

// src/remap.zig:166-278: ROI-sized output with one extra (alpha) channel.
template <typename T>
static void remapImage(T* dst, const T* src, uint32_t width, uint32_t height, int channels, const ImagePose& pose,
                       Rect roi, int jobs, double maxv) {
  uint32_t out_w = (uint32_t)(roi.right - roi.left), out_h = (uint32_t)(roi.bottom - roi.top);
  InverseTransformCache cache = initInverseTransformCache(pose, width, height);
  int dch = channels + 1;
  if (jobs <= 1 || out_h <= 32) {
    remapRows<T>(dst, src, width, height, channels, dch, roi, cache, out_w, 0, out_h, maxv);
    return;
  }
  parallelRows(out_h, jobs, [&](uint32_t s, uint32_t e) {
    remapRows<T>(dst, src, width, height, channels, dch, roi, cache, out_w, s, e, maxv);
  });
}

// src/remap.zig:585-708
struct V2 { double x, y; };
static bool isInsideEdge(V2 p, V2 a, V2 b) {
  return ((b.x - a.x) * (p.y - a.y) - (b.y - a.y) * (p.x - a.x)) >= -1e-6;
}
static V2 lineIntersection(V2 p1, V2 p2, V2 q1, V2 q2) {
  double a1 = p2.y - p1.y, b1 = p1.x - p2.x, c1 = a1 * p1.x + b1 * p1.y;
  double a2 = q2.y - q1.y, b2 = q1.x - q2.x, c2 = a2 * q1.x + b2 * q1.y;
  double det = a1 * b2 - a2 * b1;
  if (std::fabs(det) < 1e-9) return p2;
  return {(b2 * c1 - b1 * c2) / det, (a1 * c2 - a2 * c1) / det};
}
static std::vector<V2> clipPolygonToConvex(const std::vector<V2>& subject, const std::vector<V2>& clipper) {
  std::vector<V2> current = subject;
  for (size_t i = 0; i < clipper.size(); ++i) {
    V2 a = clipper[i], b = clipper[(i + 1) % clipper.size()];
    std::vector<V2> next;
    if (current.empty()) return next;
    V2 prev = current.back();
    bool prev_in = isInsideEdge(prev, a, b);
    for (V2 curr : current) {
      bool curr_in = isInsideEdge(curr, a, b);
      if (curr_in != prev_in) next.push_back(lineIntersection(prev, curr, a, b));
      if (curr_in) next.push_back(curr);
      prev = curr;
      prev_in = curr_in;
    }
    current = next;
  }
  return current;
}
static bool computeCommonOverlapRoi(const uint8_t* active, const uint32_t* widths, const uint32_t* heights,
                                    const ImagePose* poses, size_t n, Rect* out) {
  std::vector<V2> polygon;
  bool first = true;
  for (size_t i = 0; i < n; ++i) {
    if (!active[i]) continue;
    uint32_t w = widths[i], h = heights[i];
    auto fm = [&](double x, double y) {
      Point2 m = transformPoint(poses[i], x, y, w, h);
      return V2{m.x, m.y};
    };
    std::vector<V2> quad = {fm(0, 0), fm((double)(w - 1), 0), fm((double)(w - 1), (double)(h - 1)),
                            fm(0, (double)(h - 1))};
    if (first) {
      polygon = quad;
      first = false;
    } else {
      polygon = clipPolygonToConvex(polygon, quad);
      if (polygon.empty()) return false;
    }
  }
  if (polygon.empty()) return false;
  double min_x = polygon[0].x, max_x = polygon[0].x, min_y = polygon[0].y, max_y = polygon[0].y;
  for (size_t i = 1; i < polygon.size(); ++i) {
    min_x = std::min(min_x, polygon[i].x);
    max_x = std::max(max_x, polygon[i].x);
    min_y = std::min(min_y, polygon[i].y);
    max_y = std::max(max_y, polygon[i].y);
  }
  Rect r = {(int32_t)std::ceil(min_x), (int32_t)std::ceil(min_y), (int32_t)std::floor(max_x) + 1,
            (int32_t)std::floor(max_y) + 1};
  if (r.right <= r.left || r.bottom <= r.top) return false;
  *out = r;
  return true;
}

// ------------------------------------------------------------ fusion: masks
// Aligned frame = interleaved RGB or RGBA (u8/u16), row-major, no padding.
struct Frame {
  const void* pixels;
  uint32_t width, height;
  int color_channels;  // 3
  int extra_channels;  // 0 or 1
  int sample_bits;     // 8 or 16
  int stride() const { return color_channels + extra_channels; }
  uint32_t at(size_t i) const {
    return sample_bits == 8 ? ((const uint8_t*)pixels)[i] : ((const uint16_t*)pixels)[i];
  }
};

// src/fuse/grayscale.zig:4-57 (RGB colour model)
static void fillAverageFromLoaded(float* dst, const Frame& im) {
  size_t count = (size_t)im.width * im.height;
  size_t stride = im.stride();
  float denom = im.sample_bits == 8 ? (float)(3.0 * 255.0) : (float)(3.0 * 65535.0);
  for (size_t i = 0; i < count; ++i) {
    size_t b = i * stride;
    uint32_t sum = im.at(b) + im.at(b + 1) + im.at(b + 2);
    dst[i] = (float)sum / denom;
  }
}
// src/fuse/masks.zig:32-57
static void fillBinarySupport(const Frame& im, float* out) {
  size_t count = (size_t)im.width * im.height;
  if (im.extra_channels == 0) {
    for (size_t i = 0; i < count; ++i) out[i] = 1.0f;
    return;
  }
  size_t pc = im.stride(), ao = im.color_channels;
  for (size_t i = 0; i < count; ++i) out[i] = im.at(i * pc + ao) > 0 ? 1.0f : 0.0f;
}
// src/fuse/masks.zig:6-30
template <typename Real>
static void applySupportInto(const Frame& im, Real* weights) {
  if (im.extra_channels == 0) return;
  size_t count = (size_t)im.width * im.height;
  size_t pc = im.stride(), ao = im.color_channels;
  Real scale = im.sample_bits == 8 ? (Real)255.0 : (Real)65535.0;
  for (size_t i = 0; i < count; ++i) {
    Real support = (Real)im.at(i * pc + ao) / scale;
    weights[i] *= support;
  }
}
// src/fuse/masks.zig:59-84
static void accumulateBinarySupportMax(const Frame& im, float* out) {
  size_t count = (size_t)im.width * im.height;
  if (im.extra_channels == 0) {
    for (size_t i = 0; i < count; ++i) out[i] = 1.0f;
    return;
  }
  size_t pc = im.stride(), ao = im.color_channels;
  for (size_t i = 0; i < count; ++i)
    if (im.at(i * pc + ao) > 0) out[i] = 1.0f;
}

// --------------------------------------------------------- fusion: contrast
// src/fuse/contrast.zig:284-290
static float sampleStdDev(double sum, double sum_sqr, uint32_t n) {
  if (n <= 1) return 0;
  double denom = (double)(n - 1);
  double nf = (double)n;
  double variance = std::max((sum_sqr - ((sum * sum) / nf)) / denom, 0.0);
  return (float)std::sqrt(variance);
}
// src/fuse/contrast.zig:172-282
static void computeRange(const float* pixels, uint32_t width, uint32_t height, const float* support,
                         uint32_t window_size, float* weights, uint32_t start_row, uint32_t end_row) {
  if (start_row >= end_row) return;
  uint32_t border = window_size / 2;
  uint32_t first_row = std::max(start_row, border);
  uint32_t last_row_excl = std::min(end_row, height - border);
  if (first_row >= last_row_excl) return;
  int32_t W = (int32_t)width;
  size_t wu = width;
  std::vector<double> sums(wu), sums_sqr(wu);
  std::vector<uint32_t> counts(wu);
  int32_t border_i = (int32_t)border, win_i = (int32_t)window_size;
  for (size_t col = 0; col < wu; ++col) {
    double cs = 0, css = 0;
    counts[col] = 0;
    for (uint32_t yy = first_row - border; yy <= first_row + border; ++yy) {
      size_t idx = (size_t)yy * wu + col;
      if (support[idx] <= 0.0f) continue;
      double v = pixels[idx];
      cs += v;
      css += v * v;
      counts[col] += 1;
    }
    sums[col] = cs;
    sums_sqr[col] = css;
  }
  for (int32_t row = (int32_t)first_row; row < (int32_t)last_row_excl; ++row) {
    double sum = 0, sum_sqr = 0;
    uint32_t n = 0;
    for (int32_t c = 0; c < win_i; ++c) {
      sum += sums[c];
      sum_sqr += sums_sqr[c];
      n += counts[c];
    }
    int32_t x = border_i;
    size_t out = (size_t)row * wu + (size_t)border_i;
    while (true) {
      weights[out] = support[out] > 0.0f ? sampleStdDev(sum, sum_sqr, n) : 0.0f;
      if (x == W - border_i - 1) break;
      int32_t next_c = x + border_i + 1;
      size_t old_idx = (size_t)(x - border_i), next_idx = (size_t)next_c;
      sum += sums[next_idx] - sums[old_idx];
      sum_sqr += sums_sqr[next_idx] - sums_sqr[old_idx];
      n += counts[next_idx] - counts[old_idx];
      x += 1;
      out += 1;
    }
    if (row + 1 >= (int32_t)last_row_excl) continue;
    size_t rm = (size_t)(row - border_i) * wu, ad = (size_t)(row + border_i + 1) * wu;
    for (size_t c = 0; c < wu; ++c) {
      if (support[rm + c] > 0.0f) {
        double v = pixels[rm + c];
        sums[c] -= v;
        sums_sqr[c] -= v * v;
        counts[c] -= 1;
      }
      if (support[ad + c] > 0.0f) {
        double v = pixels[ad + c];
        sums[c] += v;
        sums_sqr[c] += v * v;
        counts[c] += 1;
      }
    }
  }
}
// src/fuse/contrast.zig:96-154: zero, then row ranges per worker.  The
// result depends on the worker partition (each range restarts its column
// sums), so `jobs` is a parameter.
static void computeLocalContrastWeights(const float* gray, uint32_t width, uint32_t height, const float* support,
                                        uint32_t window_size, int jobs, float* weights) {
  size_t count = (size_t)width * height;
  std::fill(weights, weights + count, 0.0f);
  if (window_size < 3 || width < window_size || height < window_size) return;
  int workers = std::min(std::max(jobs, 1), (int)height);
  if (workers <= 1) {
    computeRange(gray, width, height, support, window_size, weights, 0, height);
    return;
  }
  uint32_t rpw = (height + workers - 1) / workers;
  std::vector<std::thread> threads;
  for (int i = 0; i < workers - 1; ++i) {
    uint32_t s = (uint32_t)(i + 1) * rpw;
    uint32_t e = std::min<uint32_t>((uint32_t)(i + 2) * rpw, height);
    threads.emplace_back([=] { computeRange(gray, width, height, support, window_size, weights, s, e); });
  }
  computeRange(gray, width, height, support, window_size, weights, 0, std::min(rpw, height));
  for (auto& t : threads) t.join();
}

// ---------------------------------------------------------- fusion: pyramid
// src/fuse/pyramid.zig:163-176
static uint32_t nextLevelSize(uint32_t v) { return v > 1 ? (v + 1) / 2 : 1; }
static size_t computeLevelCount(uint32_t w, uint32_t h) {
  size_t levels = 1;
  while (w > 1 || h > 1) {
    w = nextLevelSize(w);
    h = nextLevelSize(h);
    ++levels;
  }
  return levels;
}
static const uint32_t kExactExpandMaxDim = 512;  // src/fuse/pyramid.zig:8

template <typename Real>
struct Level {
  uint32_t w = 0, h = 0;
  std::vector<Real> px;  // scalar: w*h, rgb: w*h*3 interleaved
};

static inline uint32_t clampCoord(int32_t c, uint32_t limit) {  // src/fuse/pyramid.zig:1837-1842
  if (c <= 0) return 0;
  int32_t mx = (int32_t)limit - 1;
  if (c >= mx) return (uint32_t)mx;
  return (uint32_t)c;
}
static inline float kernelWeight(int i) { return (i == 0 || i == 4) ? 1.0f : ((i == 1 || i == 3) ? 4.0f : 6.0f); }

// src/fuse/pyramid.zig:303-316
template <typename Real>
static void normalizeWeightsInto(const Real* w, const Real* norm, size_t total_images, Real* out, size_t n) {
  Real def = (Real)1.0 / (Real)total_images;
  for (size_t i = 0; i < n; ++i) out[i] = norm[i] > (Real)1e-12 ? w[i] / norm[i] : def;
}

// src/fuse/pyramid.zig:997-1042 (scalar) / 1044-1099 (rgb), NCH = 1 or 3.
template <typename Real, int NCH>
static void reduceWithSupportRows(uint32_t sw, uint32_t sh, const Real* src, const Real* support, uint32_t dw,
                                  Real* dst, Real* dst_support, uint32_t r0, uint32_t r1) {
  for (uint32_t dy = r0; dy < r1; ++dy) {
    int32_t cy = (int32_t)(dy * 2);
    for (uint32_t dx = 0; dx < dw; ++dx) {
      int32_t cx = (int32_t)(dx * 2);
      Real sum[NCH];
      for (int c = 0; c < NCH; ++c) sum[c] = 0;
      Real weight_sum = 0;
      for (int ky = 0; ky < 5; ++ky) {
        int32_t sy = cy + ky - 2;
        if (sy < 0 || sy >= (int32_t)sh) continue;
        Real wy = (Real)kernelWeight(ky);
        for (int kx = 0; kx < 5; ++kx) {
          int32_t sx = cx + kx - 2;
          if (sx < 0 || sx >= (int32_t)sw) continue;
          size_t pi = (size_t)sy * sw + (size_t)sx;
          Real s = support[pi];
          if (s <= 0) continue;
          Real weighted = wy * (Real)kernelWeight(kx) * s;
          for (int c = 0; c < NCH; ++c) sum[c] += src[pi * NCH + c] * weighted;
          weight_sum += weighted;
        }
      }
      size_t di = (size_t)dy * dw + dx;
      if (weight_sum > 0) {
        for (int c = 0; c < NCH; ++c) dst[di * NCH + c] = sum[c] / weight_sum;
        dst_support[di] = 1;
      } else {
        for (int c = 0; c < NCH; ++c) dst[di * NCH + c] = 0;
        dst_support[di] = 0;
      }
    }
  }
}

// src/fuse/pyramid.zig:1748-1775
template <typename Real>
static void horizontalExpandRgbRow(uint32_t sw, const Real* src, uint32_t sy, uint32_t dw, Real* row) {
  size_t base = (size_t)sy * sw * 3;
  for (uint32_t dx = 0; dx < dw; ++dx) {
    int32_t sx = (int32_t)(dx / 2);
    if ((dx & 1) == 0) {
      size_t b0 = base + clampCoord(sx - 1, sw) * 3, b1 = base + clampCoord(sx, sw) * 3,
             b2 = base + clampCoord(sx + 1, sw) * 3;
      for (int c = 0; c < 3; ++c) row[dx * 3 + c] = (src[b0 + c] + (Real)6.0 * src[b1 + c] + src[b2 + c]) * (Real)(1.0 / 8.0);
    } else {
      size_t b0 = base + clampCoord(sx, sw) * 3, b1 = base + clampCoord(sx + 1, sw) * 3;
      for (int c = 0; c < 3; ++c) row[dx * 3 + c] = (src[b0 + c] + src[b1 + c]) * (Real)0.5;
    }
  }
}
// src/fuse/pyramid.zig:1101-1149
template <typename Real>
static void expandRgbRows(uint32_t dw, uint32_t sw, uint32_t sh, const Real* src, Real* dst, uint32_t r0, uint32_t r1) {
  std::vector<Real> a((size_t)dw * 3), b((size_t)dw * 3), c((size_t)dw * 3);
  for (uint32_t dy = r0; dy < r1; ++dy) {
    bool even = (dy & 1) == 0;
    uint32_t by = dy / 2;
    uint32_t y0 = even ? clampCoord((int32_t)by - 1, sh) : clampCoord((int32_t)by, sh);
    uint32_t y1 = clampCoord((int32_t)by, sh);
    uint32_t y2 = even ? clampCoord((int32_t)by + 1, sh) : clampCoord((int32_t)(by + 1), sh);
    horizontalExpandRgbRow(sw, src, y0, dw, a.data());
    horizontalExpandRgbRow(sw, src, y1, dw, b.data());
    if (even) horizontalExpandRgbRow(sw, src, y2, dw, c.data());
    Real* out = dst + (size_t)dy * dw * 3;
    for (size_t i = 0; i < (size_t)dw * 3; ++i) {
      if (even) out[i] = (a[i] + (Real)6.0 * b[i] + c[i]) * (Real)(1.0 / 8.0);
      else out[i] = (a[i] + b[i]) * (Real)0.5;
    }
  }
}

// src/fuse/pyramid.zig:1167-1354: enblend-style SKIPSM expand with zero
// boundary ("no wrap") and position-dependent normalisers.
template <typename Real>
struct V3 {
  Real v[3];
};
template <typename Real> static V3<Real> vz() { return {{0, 0, 0}}; }
template <typename Real> static V3<Real> vadd(V3<Real> a, V3<Real> b) { return {{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2]}}; }
template <typename Real> static V3<Real> vmul(Real s, V3<Real> a) { return {{s * a.v[0], s * a.v[1], s * a.v[2]}}; }
template <typename Real> static V3<Real> vdiv(V3<Real> a, Real s) { return {{a.v[0] / s, a.v[1] / s, a.v[2] / s}}; }

template <typename Real>
static void expandRgbExactNoWrap(uint32_t dw, uint32_t dh, uint32_t sw, uint32_t sh, const Real* src, Real* dst) {
  std::fill(dst, dst + (size_t)dw * dh * 3, (Real)0);
  if (sw == 0 || sh == 0) return;
  typedef V3<Real> V;
  auto load = [&](size_t i) { return V{{src[i * 3], src[i * 3 + 1], src[i * 3 + 2]}}; };
  auto put = [&](uint32_t x, uint32_t y, V v) {
    size_t b = ((size_t)y * dw + x) * 3;
    dst[b] = v.v[0]; dst[b + 1] = v.v[1]; dst[b + 2] = v.v[2];
  };
  size_t swu = sw;
  std::vector<V> sc0a(swu + 1, vz<Real>()), sc0b(swu + 1, vz<Real>()), sc1a(swu + 1, vz<Real>()), sc1b(swu + 1, vz<Real>());
  bool dw_even = (dw & 1) == 0, dh_even = (dh & 1) == 0;
  const Real six = 6, four = 4;
  V zero = vz<Real>();
  {
    V sr0 = load(0), sr1 = zero;
    for (size_t sx = 1; sx < swu; ++sx) {
      V cur = load(sx);
      sc0a[sx] = vadd(vadd(sr1, vmul(six, sr0)), cur);
      sc0b[sx] = vmul(four, vadd(sr0, cur));
      sc1a[sx] = zero;
      sc1b[sx] = zero;
      sr1 = sr0;
      sr0 = cur;
    }
    sc0a[swu] = vadd(sr1, vmul(six, sr0));
    sc0b[swu] = vmul(four, sr0);
    sc1a[swu] = zero;
    sc1b[swu] = zero;
  }
  if (sh == 1) {
    if (sw == 1) {
      put(0, 0, vdiv(vadd(sc1a[1], vmul(six, sc0a[1])), (Real)36));
      if (dw_even) put(1, 0, vdiv(vadd(sc1b[1], vmul(six, sc0b[1])), (Real)24));
      if (dh_even) {
        put(0, 1, vdiv(sc0a[1], (Real)6));
        if (dw_even) put(1, 1, vdiv(sc0b[1], (Real)4));
      }
      return;
    }
    uint32_t dx = 0;
    for (size_t sx = 1; sx < swu; ++sx) {
      V o00 = vdiv(vadd(sc1a[sx], vmul(six, sc0a[sx])), (Real)(sx == 1 ? 42 : 48));
      V o10 = vdiv(vadd(sc1b[sx], vmul(six, sc0b[sx])), (Real)48);
      put(dx, 0, o00);
      dx += 1;
      put(dx, 0, o10);
      dx += 1;
      if (dh_even) {
        put(dx - 2, 1, vdiv(sc0a[sx], (Real)(sx == 1 ? 7 : 8)));
        put(dx - 1, 1, vdiv(sc0b[sx], (Real)8));
      }
    }
    size_t e = swu;
    put(dx, 0, vdiv(vadd(sc1a[e], vmul(six, sc0a[e])), (Real)49));
    if (dw_even) put(dx + 1, 0, vdiv(vadd(sc1b[e], vmul(six, sc0b[e])), (Real)28));
    if (dh_even) {
      put(dx, 1, vdiv(sc0a[e], (Real)7));
      if (dw_even) put(dx + 1, 1, vdiv(sc0b[e], (Real)4));
    }
    return;
  }
  for (size_t sy = 1; sy < (size_t)sh; ++sy) {
    V sr0 = load(sy * swu), sr1 = zero;
    uint32_t dx = 0;
    uint32_t top = (uint32_t)((sy - 1) * 2), bottom = top + 1;
    for (size_t sx = 1; sx < swu; ++sx) {
      V cur = load(sy * swu + sx);
      V o00 = vadd(sc1a[sx], vmul(six, sc0a[sx]));
      V o10 = vadd(sc1b[sx], vmul(six, sc0b[sx]));
      V o01 = sc0a[sx];
      V o11 = sc0b[sx];
      sc1a[sx] = sc0a[sx];
      sc1b[sx] = sc0b[sx];
      sc0a[sx] = vadd(vadd(sr1, vmul(six, sr0)), cur);
      sc0b[sx] = vmul(four, vadd(sr0, cur));
      sr1 = sr0;
      sr0 = cur;
      o00 = vadd(o00, sc0a[sx]);
      o10 = vadd(o10, sc0b[sx]);
      o01 = vadd(o01, sc0a[sx]);
      o11 = vadd(o11, sc0b[sx]);
      bool left = sx == 1;
      Real s00 = sy == 1 ? (left ? 49 : 56) : (left ? 56 : 64);
      Real s10 = sy == 1 ? 56 : 64;
      Real s01 = left ? 14 : 16;
      Real s11 = 16;
      put(dx, top, vdiv(o00, s00));
      dx += 1;
      put(dx, top, vdiv(o10, s10));
      dx += 1;
      put(dx - 2, bottom, vdiv(o01, s01));
      put(dx - 1, bottom, vdiv(o11, s11));
    }
    size_t e = swu;
    V o00 = vadd(sc1a[e], vmul(six, sc0a[e]));
    V o01 = sc0a[e];
    V o10 = vadd(sc1b[e], vmul(six, sc0b[e]));
    V o11 = sc0b[e];
    sc1a[e] = sc0a[e];
    sc1b[e] = sc0b[e];
    sc0a[e] = vadd(sr1, vmul(six, sr0));
    sc0b[e] = vmul(four, sr0);
    o00 = vadd(o00, sc0a[e]);
    o01 = vadd(o01, sc0a[e]);
    put(dx, top, vdiv(o00, (Real)(sy == 1 ? 49 : 56)));
    put(dx, bottom, vdiv(o01, (Real)14));
    if (dw_even) {
      o10 = vadd(o10, sc0b[e]);
      o11 = vadd(o11, sc0b[e]);
      put(dx + 1, top, vdiv(o10, (Real)(sy == 1 ? 28 : 32)));
      put(dx + 1, bottom, vdiv(o11, (Real)8));
    }
  }
  uint32_t top = (sh - 1) * 2, bottom = top + 1;
  if (sw == 1) {
    size_t sx = swu;
    put(0, top, vdiv(vadd(sc1a[sx], vmul(six, sc0a[sx])), (Real)42));
    if (dw_even) put(1, top, vdiv(vadd(sc1b[sx], vmul(six, sc0b[sx])), (Real)28));
    if (dh_even) {
      put(0, bottom, vdiv(sc0a[sx], (Real)6));
      if (dw_even) put(1, bottom, vdiv(sc0b[sx], (Real)4));
    }
    return;
  }
  uint32_t dx = 0;
  for (size_t sx = 1; sx < swu; ++sx) {
    Real s00 = sx == 1 ? 49 : 56, s10 = 56, s01 = sx == 1 ? 7 : 8, s11 = 8;
    put(dx, top, vdiv(vadd(sc1a[sx], vmul(six, sc0a[sx])), s00));
    dx += 1;
    put(dx, top, vdiv(vadd(sc1b[sx], vmul(six, sc0b[sx])), s10));
    dx += 1;
    if (dh_even) {
      put(dx - 2, bottom, vdiv(sc0a[sx], s01));
      put(dx - 1, bottom, vdiv(sc0b[sx], s11));
    }
  }
  size_t e = swu;
  put(dx, top, vdiv(vadd(sc1a[e], vmul(six, sc0a[e])), (Real)49));
  if (dw_even) put(dx + 1, top, vdiv(vadd(sc1b[e], vmul(six, sc0b[e])), (Real)28));
  if (dh_even) {
    put(dx, bottom, vdiv(sc0a[e], (Real)7));
    if (dw_even) put(dx + 1, bottom, vdiv(sc0b[e], (Real)4));
  }
}

// src/fuse/pyramid.zig:849-909
template <typename Real>
static void expandRgb(uint32_t dw, uint32_t dh, uint32_t sw, uint32_t sh, const Real* src, Real* dst, int jobs) {
  if (std::max(dw, dh) <= kExactExpandMaxDim) {
    expandRgbExactNoWrap<Real>(dw, dh, sw, sh, src, dst);
    return;
  }
  parallelRows(dh, jobs, [&](uint32_t s, uint32_t e) { expandRgbRows<Real>(dw, sw, sh, src, dst, s, e); });
}

// src/fuse/pyramid.zig:34-62 (Accumulator) and 69-148 (Workspace)
template <typename Real>
struct Pyramid {
  std::vector<Level<Real>> acc;           // RGB
  std::vector<Level<Real>> mask, mask_support, gauss, image_support, expanded;
  void init(uint32_t w, uint32_t h) {
    size_t L = computeLevelCount(w, h);
    acc.resize(L); mask.resize(L); mask_support.resize(L); gauss.resize(L); image_support.resize(L);
    expanded.resize(L > 0 ? L - 1 : 0);
    for (size_t i = 0; i < L; ++i) {
      size_t n = (size_t)w * h;
      acc[i].w = mask[i].w = mask_support[i].w = gauss[i].w = image_support[i].w = w;
      acc[i].h = mask[i].h = mask_support[i].h = gauss[i].h = image_support[i].h = h;
      acc[i].px.assign(n * 3, (Real)0);
      mask[i].px.assign(n, 0); mask_support[i].px.assign(n, 0);
      gauss[i].px.assign(n * 3, 0); image_support[i].px.assign(n, 0);
      if (i + 1 < L) { expanded[i].w = w; expanded[i].h = h; expanded[i].px.assign(n * 3, 0); }
      w = nextLevelSize(w);
      h = nextLevelSize(h);
    }
  }
};

// src/fuse/pyramid.zig:190-204, 384-416, 489-542, 572-639, 1506-1649
template <typename Real>
static void accumulateImage(const Frame& im, const Real* normalized_mask, const float* union_support, Pyramid<Real>& P,
                            int jobs) {
  size_t L = P.acc.size();
  size_t n0 = (size_t)im.width * im.height;
  // buildMaskGaussianPyramidInto
  std::copy(normalized_mask, normalized_mask + n0, P.mask[0].px.begin());
  for (size_t i = 0; i < n0; ++i) P.mask_support[0].px[i] = (Real)union_support[i];
  for (size_t l = 1; l < L; ++l) {
    auto& pv = P.mask[l - 1]; auto& ps = P.mask_support[l - 1];
    auto& nv = P.mask[l]; auto& ns = P.mask_support[l];
    parallelRows(nv.h, jobs, [&](uint32_t s, uint32_t e) {
      reduceWithSupportRows<Real, 1>(pv.w, pv.h, pv.px.data(), ps.px.data(), nv.w, nv.px.data(), ns.px.data(), s, e);
    });
  }
  // buildAndAccumulateImagePyramidInto: fillRgbBase + fillBinarySupport
  {
    size_t sc = im.stride();
    parallelRows(im.height, n0 >= 262144 ? jobs : 1, [&](uint32_t r0, uint32_t r1) {  // fillRgbBase
      for (size_t i = (size_t)r0 * im.width; i < (size_t)r1 * im.width; ++i)
        for (int c = 0; c < 3; ++c) P.gauss[0].px[i * 3 + c] = (Real)im.at(i * sc + c);
    });
    std::vector<float> sup(n0);
    fillBinarySupport(im, sup.data());
    for (size_t i = 0; i < n0; ++i) P.image_support[0].px[i] = (Real)sup[i];
  }
  for (size_t l = 1; l < L; ++l) {
    auto& pv = P.gauss[l - 1]; auto& ps = P.image_support[l - 1];
    auto& nv = P.gauss[l]; auto& ns = P.image_support[l];
    parallelRows(nv.h, jobs, [&](uint32_t s, uint32_t e) {
      reduceWithSupportRows<Real, 3>(pv.w, pv.h, pv.px.data(), ps.px.data(), nv.w, nv.px.data(), ns.px.data(), s, e);
    });
  }
  for (size_t l = 0; l + 1 < L; ++l) {
    auto& cur = P.gauss[l]; auto& nxt = P.gauss[l + 1]; auto& ex = P.expanded[l];
    expandRgb<Real>(cur.w, cur.h, nxt.w, nxt.h, nxt.px.data(), ex.px.data(), jobs);
    const Real* m = P.mask[l].px.data();
    Real* dst = P.acc[l].px.data();
    size_t n = (size_t)cur.w * cur.h;
    // accumulateLapRowsSequential, src/fuse/pyramid.zig:1480-1504 (row-parallel
    // above 262144 pixels like src/fuse/pyramid.zig:1463-1467)
    parallelRows(cur.h, n >= 262144 ? jobs : 1, [&](uint32_t r0, uint32_t r1) {
      for (size_t i = (size_t)r0 * cur.w; i < (size_t)r1 * cur.w; ++i) {
        Real wgt = m[i];
        for (int c = 0; c < 3; ++c) {
          Real lap = cur.px[i * 3 + c] - ex.px[i * 3 + c];
          dst[i * 3 + c] += lap * wgt;
        }
      }
    });
  }
  {  // accumulateGaussianRowsSequential, src/fuse/pyramid.zig:1506-1529
    auto& g = P.gauss[L - 1];
    const Real* m = P.mask[L - 1].px.data();
    Real* dst = P.acc[L - 1].px.data();
    size_t n = (size_t)g.w * g.h;
    for (size_t i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) dst[i * 3 + c] += g.px[i * 3 + c] * m[i];
  }
}

// src/fuse/pyramid.zig:223-269: collapse a copy of the accumulator, then
// quantise: trunc(clamp(v + 0.5, 0, max)).  Writes interleaved RGB.
template <typename Real>
static void collapse(const Pyramid<Real>& P, int sample_bits, void* out, Real* base_out, int jobs) {
  std::vector<Level<Real>> c = P.acc;
  for (size_t li = c.size(); li > 1;) {
    --li;
    auto& child = c[li];
    auto& parent = c[li - 1];
    std::vector<Real> ex((size_t)parent.w * parent.h * 3);
    expandRgb<Real>(parent.w, parent.h, child.w, child.h, child.px.data(), ex.data(), jobs);
    for (size_t i = 0; i < ex.size(); ++i) parent.px[i] += ex[i];
  }
  const auto& base = c[0];
  double maxv = sample_bits == 8 ? 255.0 : 65535.0;
  for (size_t i = 0; i < base.px.size(); ++i) {
    Real v = base.px[i] + (Real)0.5;
    Real cl = std::max((Real)0.0, std::min(v, (Real)maxv));
    if (sample_bits == 8) ((uint8_t*)out)[i] = (uint8_t)cl;
    else ((uint16_t*)out)[i] = (uint16_t)cl;
    if (base_out) base_out[i] = base.px[i];
  }
}

// Weight map for one aligned frame: src/stack/pipeline.zig:653-671 then
// masks.applySupportInto (src/stack/pipeline.zig:467).
static void weightMap(const Frame& im, uint32_t window, int jobs, std::vector<float>& gray, std::vector<float>& sup,
                      std::vector<float>& w) {
  size_t n = (size_t)im.width * im.height;
  gray.resize(n); sup.resize(n); w.resize(n);
  parallelRows(im.height, jobs, [&](uint32_t r0, uint32_t r1) {
    Frame band = im;
    size_t off = (size_t)r0 * im.width * im.stride() * (im.sample_bits == 8 ? 1 : 2);
    band.pixels = (const uint8_t*)im.pixels + off;
    band.height = r1 - r0;
    fillAverageFromLoaded(gray.data() + (size_t)r0 * im.width, band);
    fillBinarySupport(band, sup.data() + (size_t)r0 * im.width);
  });
  computeLocalContrastWeights(gray.data(), im.width, im.height, sup.data(), window, jobs, w.data());
  parallelRows(im.height, jobs, [&](uint32_t r0, uint32_t r1) {
    Frame band = im;
    size_t off = (size_t)r0 * im.width * im.stride() * (im.sample_bits == 8 ? 1 : 2);
    band.pixels = (const uint8_t*)im.pixels + off;
    band.height = r1 - r0;
    applySupportInto<float>(band, w.data() + (size_t)r0 * im.width);
  });
}

}  // namespace oracle

// ===================================================================== C API
using namespace oracle;

extern "C" {

// Pose record layout shared with the C-ABI (15 doubles, ImagePose order).
struct or_pose { double v[15]; };
static ImagePose toPose(const or_pose* p) {
  ImagePose q;
  const double* v = p->v;
  q.yaw = v[0]; q.pitch = v[1]; q.roll = v[2]; q.hfov_delta = v[3];
  q.trans_x = v[4]; q.trans_y = v[5]; q.trans_z = v[6];
  q.translation_plane_yaw = v[7]; q.translation_plane_pitch = v[8];
  q.radial_a = v[9]; q.radial_b = v[10]; q.radial_c = v[11];
  q.center_shift_x = v[12]; q.center_shift_y = v[13]; q.base_hfov_degrees = v[14];
  return q;
}

// inverse map of one point (src/optimize.zig:3593); used to pin the
// homography composition of the CUDA path.
void oracle_inverse_point(const or_pose* pose, uint32_t w, uint32_t h, double ox, double oy, double* sx, double* sy) {
  InverseTransformCache c = initInverseTransformCache(toPose(pose), w, h);
  Point2 p;
  if (!c.basic_rectilinear && !c.has_translation) {
    // per-pixel formula of remapU8RowsNoTranslationLens without the
    // row-incremental accumulation
    Vec3 pano = {ox - c.dest_center_x, oy - c.dest_center_y, -c.dest_focal};
    Vec3 l = matrixMul(c.world_to_local, pano);
    double denom = -l.z;
    if (std::fabs(denom) < 1e-12) { *sx = -1; *sy = -1; return; }
    double rx = c.image_focal * (l.x / denom) + c.center_shift_x;
    double ry = c.image_focal * (l.y / denom) + c.center_shift_y;
    bool radial = c.radial_a != 0.0 || c.radial_b != 0.0 || c.radial_c != 0.0;
    p = radial ? undistortSourcePoint(c, rx, ry) : Point2{c.src_center_x + rx, c.src_center_y + ry};
  } else {
    p = inverseTransformPointCached(c, ox, oy);
  }
  *sx = p.x;
  *sy = p.y;
}

void oracle_forward_point(const or_pose* pose, uint32_t w, uint32_t h, double x, double y, double* ox, double* oy) {
  Point2 p = transformPoint(toPose(pose), x, y, w, h);
  *ox = p.x;
  *oy = p.y;
}

// src/remap.zig:585-633.  Returns 1 with *out set, or 0 when there is no overlap.
int oracle_compute_roi(const or_pose* poses, const uint32_t* widths, const uint32_t* heights, const uint8_t* active,
                       size_t n, int32_t* out4) {
  std::vector<ImagePose> ps(n);
  for (size_t i = 0; i < n; ++i) ps[i] = toPose(&poses[i]);
  Rect r = {0, 0, 0, 0};
  if (!computeCommonOverlapRoi(active, widths, heights, ps.data(), n, &r)) return 0;
  out4[0] = r.left; out4[1] = r.top; out4[2] = r.right; out4[3] = r.bottom;
  return 1;
}

// src/remap.zig:166-278.  roi == NULL means the full frame.  dst holds
// (channels + 1) samples per pixel.
void oracle_remap(const void* src, uint32_t width, uint32_t height, int channels, int sample_bits, const or_pose* pose,
                  const int32_t* roi4, int jobs, void* dst) {
  Rect roi = roi4 ? Rect{roi4[0], roi4[1], roi4[2], roi4[3]} : Rect{0, 0, (int32_t)width, (int32_t)height};
  if (sample_bits == 8)
    remapImage<uint8_t>((uint8_t*)dst, (const uint8_t*)src, width, height, channels, toPose(pose), roi, jobs, 255.0);
  else
    remapImage<uint16_t>((uint16_t*)dst, (const uint16_t*)src, width, height, channels, toPose(pose), roi, jobs, 65535.0);
}

// Weight map of one aligned frame (gray, support, contrast, alpha): the
// pass-1 per-frame product.
void oracle_weight_map(const void* pixels, uint32_t width, uint32_t height, int extra_channels, int sample_bits,
                       uint32_t window, int jobs, float* out) {
  Frame im{pixels, width, height, 3, extra_channels, sample_bits};
  std::vector<float> g, s, w;
  weightMap(im, window, jobs, g, s, w);
  std::copy(w.begin(), w.end(), out);
}

void oracle_fill_average(const void* pixels, uint32_t width, uint32_t height, int extra_channels, int sample_bits,
                         float* out) {
  Frame im{pixels, width, height, 3, extra_channels, sample_bits};
  fillAverageFromLoaded(out, im);
}

float oracle_sample_stddev(double sum, double sum_sqr, uint32_t n) { return sampleStdDev(sum, sum_sqr, n); }

void oracle_normalize_weights(const float* w, const float* norm, size_t total_images, float* out, size_t n) {
  normalizeWeightsInto<float>(w, norm, total_images, out, n);
}

size_t oracle_level_count(uint32_t w, uint32_t h) { return computeLevelCount(w, h); }

void oracle_reduce_rgb_with_support(uint32_t sw, uint32_t sh, const float* src, const float* support, float* dst,
                                    float* dst_support) {
  uint32_t dw = nextLevelSize(sw), dh = nextLevelSize(sh);
  reduceWithSupportRows<float, 3>(sw, sh, src, support, dw, dst, dst_support, 0, dh);
}
void oracle_reduce_scalar_with_support(uint32_t sw, uint32_t sh, const float* src, const float* support, float* dst,
                                       float* dst_support) {
  uint32_t dw = nextLevelSize(sw), dh = nextLevelSize(sh);
  reduceWithSupportRows<float, 1>(sw, sh, src, support, dw, dst, dst_support, 0, dh);
}
// plain clamped five-tap reduce (reduceRgbRowsSequential, src/fuse/pyramid.zig:950-995):
// the reference's uniform-image known-answer test and the Laplacian pyramids
// of the hybrid method (buildImageLaplacianPyramid, src/fuse/pyramid.zig:418-488).
void oracle_reduce_rgb_plain(uint32_t sw, uint32_t sh, const float* src, float* dst) {
  uint32_t dw = nextLevelSize(sw), dh = nextLevelSize(sh);
  std::vector<float> rows(5 * (size_t)dw * 3);
  auto hrow = [&](uint32_t sy, float* out) {  // horizontalReduceRgbRow, src/fuse/pyramid.zig:1725-1746
    size_t base = (size_t)sy * sw * 3;
    for (uint32_t dx = 0; dx < dw; ++dx) {
      int32_t sx = (int32_t)(dx * 2);
      size_t b0 = base + clampCoord(sx - 2, sw) * 3, b1 = base + clampCoord(sx - 1, sw) * 3,
             b2 = base + clampCoord(sx, sw) * 3, b3 = base + clampCoord(sx + 1, sw) * 3,
             b4 = base + clampCoord(sx + 2, sw) * 3;
      for (int c = 0; c < 3; ++c)
        out[dx * 3 + c] = (src[b0 + c] + 4.0f * src[b1 + c] + 6.0f * src[b2 + c] + 4.0f * src[b3 + c] + src[b4 + c]) *
                          (1.0f / 16.0f);
    }
  };
  for (uint32_t dy = 0; dy < dh; ++dy) {
    int32_t cy = (int32_t)(dy * 2);
    for (int k = 0; k < 5; ++k) hrow(clampCoord(cy + k - 2, sh), rows.data() + (size_t)k * dw * 3);
    const float* r[5];
    for (int k = 0; k < 5; ++k) r[k] = rows.data() + (size_t)k * dw * 3;
    for (size_t i = 0; i < (size_t)dw * 3; ++i)
      dst[(size_t)dy * dw * 3 + i] = (r[0][i] + 4.0f * r[1][i] + 6.0f * r[2][i] + 4.0f * r[3][i] + r[4][i]) * (1.0f / 16.0f);
  }
}
void oracle_expand_rgb(uint32_t dw, uint32_t dh, uint32_t sw, uint32_t sh, const float* src, float* dst) {
  expandRgb<float>(dw, dh, sw, sh, src, dst, 1);
}

// Full pyramid-contrast fusion of aligned RGB(A) frames: the fuse-only
// driver src/fuse/pipeline.zig:254-445 with collapse
// src/fuse/pipeline.zig:180-194.  frames[k] points at frame k (same size,
// same layout).  precision 32 = reference f32 arithmetic, 64 = FP64
// evaluation of the same pyramid.  base_out (optional, width*height*3
// doubles) receives the collapsed base level before quantisation.
int oracle_fuse_aligned(const void* const* frames, size_t count, uint32_t width, uint32_t height, int extra_channels,
                        int sample_bits, uint32_t window, int jobs, int precision, void* out_rgb, double* base_out) {
  if (count == 0) return -1;
  size_t n = (size_t)width * height;
  std::vector<float> gray, sup, w;
  std::vector<float> norm32(n, 0.0f), uni(n, 0.0f);
  std::vector<double> norm64(n, 0.0);
  auto frame = [&](size_t k) { return Frame{frames[k], width, height, 3, extra_channels, sample_bits}; };
  // pass 1 (src/fuse/pipeline.zig:292-334)
  for (size_t k = 0; k < count; ++k) {
    Frame im = frame(k);
    if (precision == 32) {
      weightMap(im, window, jobs, gray, sup, w);
      accumulateBinarySupportMax(im, uni.data());
      parallelRows(height, jobs, [&](uint32_t r0, uint32_t r1) {
        for (size_t i = (size_t)r0 * width; i < (size_t)r1 * width; ++i) norm32[i] += w[i];
      });
    } else {
      gray.resize(n); sup.resize(n); w.resize(n);
      fillAverageFromLoaded(gray.data(), im);
      fillBinarySupport(im, sup.data());
      computeLocalContrastWeights(gray.data(), width, height, sup.data(), window, jobs, w.data());
      std::vector<double> wd(w.begin(), w.end());
      applySupportInto<double>(im, wd.data());
      accumulateBinarySupportMax(im, uni.data());
      for (size_t i = 0; i < n; ++i) norm64[i] += wd[i];
    }
  }
  std::vector<double> base;
  if (precision == 32) {
    Pyramid<float> P;
    P.init(width, height);
    std::vector<float> m(n);
    for (size_t k = 0; k < count; ++k) {  // pass 2 (src/fuse/pipeline.zig:389-420)
      Frame im = frame(k);
      weightMap(im, window, jobs, gray, sup, w);
      parallelRows(height, jobs, [&](uint32_t r0, uint32_t r1) {
        size_t b = (size_t)r0 * width, e = (size_t)r1 * width;
        normalizeWeightsInto<float>(w.data() + b, norm32.data() + b, count, m.data() + b, e - b);
      });
      accumulateImage<float>(im, m.data(), uni.data(), P, jobs);
    }
    std::vector<float> b(n * 3);
    collapse<float>(P, sample_bits, out_rgb, b.data(), jobs);
    if (base_out) for (size_t i = 0; i < n * 3; ++i) base_out[i] = b[i];
  } else {
    Pyramid<double> P;
    P.init(width, height);
    std::vector<double> m(n), wd(n);
    for (size_t k = 0; k < count; ++k) {
      Frame im = frame(k);
      gray.resize(n); sup.resize(n); w.resize(n);
      fillAverageFromLoaded(gray.data(), im);
      fillBinarySupport(im, sup.data());
      computeLocalContrastWeights(gray.data(), width, height, sup.data(), window, jobs, w.data());
      for (size_t i = 0; i < n; ++i) wd[i] = w[i];
      applySupportInto<double>(im, wd.data());
      normalizeWeightsInto<double>(wd.data(), norm64.data(), count, m.data(), n);
      accumulateImage<double>(im, m.data(), uni.data(), P, jobs);
    }
    std::vector<double> b(n * 3);
    collapse<double>(P, sample_bits, out_rgb, b.data(), jobs);
    if (base_out) for (size_t i = 0; i < n * 3; ++i) base_out[i] = b[i];
  }
  return 0;
}

// Stack path: remap each active frame through its pose into the ROI, then
// fuse (src/stack/pipeline.zig:361-605).  Frames are interleaved RGB
// (channels = 3) of one size.  roi4 == NULL means the full frame.
int oracle_stack_fuse(const void* const* sources, size_t count, uint32_t width, uint32_t height, int sample_bits,
                      const or_pose* poses, const int32_t* roi4, uint32_t window, int jobs, int precision,
                      void* out_rgb, double* base_out) {
  Rect roi = roi4 ? Rect{roi4[0], roi4[1], roi4[2], roi4[3]} : Rect{0, 0, (int32_t)width, (int32_t)height};
  uint32_t ow = (uint32_t)(roi.right - roi.left), oh = (uint32_t)(roi.bottom - roi.top);
  size_t bytes = (size_t)ow * oh * 4 * (sample_bits == 8 ? 1 : 2);
  std::vector<std::vector<uint8_t>> remapped(count, std::vector<uint8_t>(bytes));
  std::vector<const void*> ptrs(count);
  for (size_t k = 0; k < count; ++k) {
    oracle_remap(sources[k], width, height, 3, sample_bits, &poses[k], roi4, jobs, remapped[k].data());
    ptrs[k] = remapped[k].data();
  }
  return oracle_fuse_aligned(ptrs.data(), count, ow, oh, 1, sample_bits, window, jobs, precision, out_rgb, base_out);
}


// blend.updateWinners (src/fuse/blend.zig:188-289) over n pixels of one image
// (3 colour channels + extra_channels, u8 or u16): where the weight times the
// alpha support (effectiveWeightU8/U16: f32(alpha) / 255 or / 65535) is
// strictly larger than best, it becomes best and the pixel's colour is
// copied into out (3 samples per pixel).
void oracle_update_winners(const void* image, size_t n, int extra_channels, int sample_bits, const float* weights,
                           float* best, void* out) {
  const size_t st = 3 + (size_t)extra_channels;
  for (size_t i = 0; i < n; ++i) {
    float wgt = weights[i];
    if (extra_channels) {
      const float al = sample_bits == 8 ? (float)((const uint8_t*)image)[i * st + 3]
                                        : (float)((const uint16_t*)image)[i * st + 3];
      wgt = wgt * (al / (sample_bits == 8 ? 255.0f : 65535.0f));
    }
    if (wgt <= best[i]) continue;
    best[i] = wgt;
    for (int c = 0; c < 3; ++c) {
      if (sample_bits == 8) ((uint8_t*)out)[i * 3 + c] = ((const uint8_t*)image)[i * st + c];
      else ((uint16_t*)out)[i * 3 + c] = ((const uint16_t*)image)[i * st + c];
    }
  }
}

// mergeHybridImages (src/fuse/pyramid.zig:271-301) of two interleaved RGB
// images (u8 or u16): Laplacian pyramids by buildImageLaplacianPyramid
// (src/fuse/pyramid.zig:418-488: plain clamped REDUCE, expandRgb), levels
// [hard_start, hard_start + hard_count) mixed as soft + (hard - soft) * mix,
// the others soft's, collapsed and quantised (base_out: the collapsed base).
void oracle_hybrid_merge(const void* soft, const void* hard, uint32_t ow, uint32_t oh, int sample_bits,
                         uint32_t hard_start, uint32_t hard_count, float mix, int jobs, void* out_rgb,
                         double* base_out) {
  const size_t n = (size_t)ow * oh;
  const size_t L = computeLevelCount(ow, oh);
  auto laplacians = [&](const void* img) {
    std::vector<Level<float>> g(L);
    g[0].w = ow;
    g[0].h = oh;
    g[0].px.resize(n * 3);
    for (size_t i = 0; i < n * 3; ++i)
      g[0].px[i] = sample_bits == 8 ? (float)((const uint8_t*)img)[i] : (float)((const uint16_t*)img)[i];
    for (size_t l = 1; l < L; ++l) {
      g[l].w = nextLevelSize(g[l - 1].w);
      g[l].h = nextLevelSize(g[l - 1].h);
      g[l].px.resize((size_t)g[l].w * g[l].h * 3);
      oracle_reduce_rgb_plain(g[l - 1].w, g[l - 1].h, g[l - 1].px.data(), g[l].px.data());
    }
    for (size_t l = 0; l + 1 < L; ++l) {
      std::vector<float> ex(g[l].px.size());
      expandRgb<float>(g[l].w, g[l].h, g[l + 1].w, g[l + 1].h, g[l + 1].px.data(), ex.data(), jobs);
      for (size_t i = 0; i < ex.size(); ++i) g[l].px[i] = g[l].px[i] - ex[i];
    }
    return g;
  };
  std::vector<Level<float>> ls = laplacians(soft), lh = laplacians(hard);
  Pyramid<float> P;
  P.init(ow, oh);
  const size_t hs = std::min<size_t>(hard_start, L), he = std::min<size_t>(hs + hard_count, L);
  for (size_t l = 0; l < L; ++l) {
    auto& dst = P.acc[l].px;
    for (size_t i = 0; i < dst.size(); ++i)
      dst[i] = (l >= hs && l < he) ? ls[l].px[i] + (lh[l].px[i] - ls[l].px[i]) * mix : ls[l].px[i];
  }
  std::vector<float> b(n * 3);
  collapse<float>(P, sample_bits, out_rgb, b.data(), jobs);
  if (base_out) for (size_t i = 0; i < n * 3; ++i) base_out[i] = b[i];
}

// hybrid-pyramid-contrast, stack path (src/stack/pipeline.zig:177-236): the
// pyramid-contrast output ("soft"), the hardmask-contrast output ("hard":
// runRemappedSinglePass with blend.updateWinners, src/stack/pipeline.zig:
// 245-310, src/fuse/blend.zig:188-289 -- per pixel the colour of the first
// frame, in order, whose weight x alpha/max is largest; best weights start at
// -inf) and mergeHybridImages (src/fuse/pyramid.zig:271-301): Laplacian
// pyramids of both images (plain clamped REDUCE, expandRgb), levels
// [hard_start, hard_start + hard_count) mixed as soft + (hard - soft) * mix,
// the others soft's, collapsed and quantised.  hard_out (optional) receives
// the hard image.
int oracle_stack_fuse_hybrid(const void* const* sources, size_t count, uint32_t width, uint32_t height,
                             int sample_bits, const or_pose* poses, const int32_t* roi4, uint32_t window, int jobs,
                             uint32_t hard_start, uint32_t hard_count, float mix, void* out_rgb, double* base_out,
                             void* hard_out) {
  if (count == 0) return -1;
  Rect roi = roi4 ? Rect{roi4[0], roi4[1], roi4[2], roi4[3]} : Rect{0, 0, (int32_t)width, (int32_t)height};
  const uint32_t ow = (uint32_t)(roi.right - roi.left), oh = (uint32_t)(roi.bottom - roi.top);
  const size_t n = (size_t)ow * oh, bps = sample_bits == 8 ? 1 : 2;
  std::vector<uint8_t> soft(n * 3 * bps), hard(n * 3 * bps, 0);
  int rc = oracle_stack_fuse(sources, count, width, height, sample_bits, poses, roi4, window, jobs, 32, soft.data(),
                             nullptr);
  if (rc != 0) return rc;
  std::vector<float> best(n, -INFINITY);
  std::vector<uint8_t> remapped(n * 4 * bps);
  std::vector<float> gray, sup, w;
  for (size_t k = 0; k < count; ++k) {
    oracle_remap(sources[k], width, height, 3, sample_bits, &poses[k], roi4, jobs, remapped.data());
    Frame im{remapped.data(), ow, oh, 3, 1, sample_bits};
    // computeWeightMapForRemapped: the contrast weights before applySupport
    gray.resize(n); sup.resize(n); w.resize(n);
    fillAverageFromLoaded(gray.data(), im);
    fillBinarySupport(im, sup.data());
    computeLocalContrastWeights(gray.data(), ow, oh, sup.data(), window, jobs, w.data());
    oracle_update_winners(remapped.data(), n, 1, sample_bits, w.data(), best.data(), hard.data());
  }
  if (hard_out) std::memcpy(hard_out, hard.data(), hard.size());
  oracle_hybrid_merge(soft.data(), hard.data(), ow, oh, sample_bits, hard_start, hard_count, mix, jobs, out_rgb,
                      base_out);
  return 0;
}


// The pass-2 stages of one frame and the collapse, over an accumulator
// pyramid held by the caller (levels 0 .. L-1 of interleaved RGB f32,
// concatenated): accumulateImage (src/fuse/pyramid.zig:190-204, the mask and
// image pyramids of the frame and the weighted blend) and
// collapseToImageWithJobs (src/fuse/pyramid.zig:223-269).  They let a test
// split a stack over several processes the way the library's phase entry
// points do.
size_t oracle_pyramid_floats(uint32_t width, uint32_t height) {
  size_t n = 0;
  for (size_t l = 0, L = computeLevelCount(width, height); l < L; ++l) {
    n += (size_t)width * height * 3;
    width = nextLevelSize(width);
    height = nextLevelSize(height);
  }
  return n;
}

static void load_acc(Pyramid<float>& P, const float* acc) {
  size_t off = 0;
  for (auto& lv : P.acc) {
    std::copy(acc + off, acc + off + lv.px.size(), lv.px.begin());
    off += lv.px.size();
  }
}

void oracle_pyramid_accumulate(const void* frame, uint32_t width, uint32_t height, int extra_channels,
                               int sample_bits, const float* normalized_mask, const float* union_support, float* acc,
                               int jobs) {
  Pyramid<float> P;
  P.init(width, height);
  load_acc(P, acc);
  accumulateImage<float>(Frame{frame, width, height, 3, extra_channels, sample_bits}, normalized_mask, union_support,
                         P, jobs);
  size_t off = 0;
  for (auto& lv : P.acc) {
    std::copy(lv.px.begin(), lv.px.end(), acc + off);
    off += lv.px.size();
  }
}

void oracle_pyramid_collapse(const float* acc, uint32_t width, uint32_t height, int sample_bits, void* out_rgb,
                             double* base_out, int jobs) {
  Pyramid<float> P;
  P.init(width, height);
  load_acc(P, acc);
  std::vector<float> b((size_t)width * height * 3);
  collapse<float>(P, sample_bits, out_rgb, b.data(), jobs);
  if (base_out) for (size_t i = 0; i < b.size(); ++i) base_out[i] = b[i];
}

}  // extern "C"
