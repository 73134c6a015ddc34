// CPU renderer of the synthetic focus stacks (TEST INFRASTRUCTURE ONLY).
//
// bench.py's CPU legs (the --impl reference arm and the cpu_baseline leg)
// time the oracle on frames of the same scene recipe as the library's device
// generator, without loading the library: this file restates that recipe on
// the host.
//
// Scene (aligned-frame coordinates X, Y):
//   T(X, Y; sigma) = sum_i A_i exp(-sigma^2 w_i^2 / 2) sin(w_i (X cos t_i + Y sin t_i) + p_i)
// with 64 components, A_i ~ U(5, 30), t_i ~ U(0, pi), p_i ~ U(0, 2 pi) and
// w_i in [0.05, 1.2] rad/px on an even grid of w_i^2; the sum is scaled by
// 0.28.  Depth d in [0, 1] from 6 low-frequency cosines; frame k focuses at
// z_k = k / (F - 1) with blur sigma_k = min(|d - z_k| * s, cap) (s = cap = 3
// for the small scene, 8 for the production scene).  Per-channel gain and
// offset, N(0, 4^2) noise, rounded and clamped to u8.  Source pixel (x, y)
// of frame k shows the scene at the forward map of its pose (the oracle's
// restatement of the reference's transformPoint), so that remapping with the
// pose realigns it.  Poses: frame 0 identity; others roll U(-r, r) deg, yaw
// and pitch atan(shift / f) with shift U(-s, s) px, focal ratio
// 1 + U(-0.005, 0.005).  Random draws use the same SplitMix64 sequence as the
// device generator, so scene parameters and poses are identical to it; pixel
// values agree to the rounding of the float arithmetic (noise, sin, exp).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

extern "C" {
struct or_pose { double v[15]; };
void oracle_forward_point(const or_pose* pose, uint32_t w, uint32_t h, double x, double y, double* ox, double* oy);
}

namespace {

constexpr int kComp = 64;
constexpr int kDepthTerms = 6;
constexpr float kContrastGain = 0.28f;
constexpr int kRun = 16;
const double kPi = 3.14159265358979323846;

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uni(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }
double uni(uint64_t& s, double lo, double hi) { return lo + (hi - lo) * uni(s); }

struct SceneConfig {
  double blur_scale, blur_cap, shift, roll_deg;
};
SceneConfig scene_config(int scene) {
  if (scene == 0) return {3.0, 3.0, 20.0, 0.2};
  return {8.0, 8.0, 60.0, 0.3};
}

struct Scene {
  float kx[kComp], ky[kComp], p0[kComp], amp[kComp];
  float w2_0, dw2;
  float dkx[kDepthTerms], dky[kDepthTerms], dp[kDepthTerms], da[kDepthTerms];
  float dnorm;
  float gain[3], offset[3];
  float blur_scale, blur_cap, z;
  uint32_t seed_lo, seed_hi, frame;
};

// Pose fields in fs_pose / ImagePose order: yaw, pitch, roll, hfov_delta, ...,
// base_hfov_degrees (index 14).
void make_pose(uint64_t seed, int scene, uint32_t width, uint32_t frame, or_pose* p) {
  std::memset(p, 0, sizeof(*p));
  p->v[14] = 50.0;
  if (frame == 0) return;
  const SceneConfig cfg = scene_config(scene);
  uint64_t s = seed * 0x2545F4914F6CDD1Dull + 0x1000ull * (frame + 1);
  const double f = ((double)width * 0.5) / std::tan(p->v[14] * kPi / 360.0);
  const double sx = uni(s, -cfg.shift, cfg.shift), sy = uni(s, -cfg.shift, cfg.shift);
  p->v[2] = uni(s, -cfg.roll_deg, cfg.roll_deg) * kPi / 180.0;
  p->v[0] = std::atan(sx / f);
  p->v[1] = std::atan(sy / f);
  const double ratio = 1.0 + uni(s, -0.005, 0.005);
  const double hfov = 2.0 * std::atan((double)width * 0.5 / (f * ratio)) * 180.0 / kPi;
  p->v[3] = hfov - p->v[14];
}

Scene make_scene(uint64_t seed, int scene, uint32_t width, uint32_t height, uint32_t frame, uint32_t frame_count) {
  const SceneConfig cfg = scene_config(scene);
  Scene sc;
  std::memset(&sc, 0, sizeof(sc));
  uint64_t s = seed * 0x9E3779B97F4A7C15ull + 17;
  const double wmin = 0.05, wmax = 1.2;
  sc.w2_0 = (float)(wmin * wmin);
  sc.dw2 = (float)((wmax * wmax - wmin * wmin) / (kComp - 1));
  int order[kComp];
  for (int i = 0; i < kComp; ++i) order[i] = i;
  for (int i = kComp - 1; i > 0; --i) {
    const int j = (int)(splitmix(s) % (uint64_t)(i + 1));
    const int t = order[i];
    order[i] = order[j];
    order[j] = t;
  }
  double A[kComp], T[kComp], P[kComp];
  for (int i = 0; i < kComp; ++i) {
    A[i] = uni(s, 5.0, 30.0);
    T[i] = uni(s, 0.0, kPi);
    P[i] = uni(s, 0.0, 2.0 * kPi);
  }
  for (int i = 0; i < kComp; ++i) {
    const int o = order[i];
    const double w = std::sqrt(wmin * wmin + (wmax * wmax - wmin * wmin) * i / (kComp - 1.0));
    sc.kx[i] = (float)(w * std::cos(T[o]) / (2.0 * kPi));
    sc.ky[i] = (float)(w * std::sin(T[o]) / (2.0 * kPi));
    sc.p0[i] = (float)(P[o] / (2.0 * kPi));
    sc.amp[i] = (float)A[o];
  }
  double dsum = 0.0;
  for (int t = 0; t < kDepthTerms; ++t) {
    const double fx = uni(s, 0.3, 2.0), fy = uni(s, 0.3, 2.0);
    const double ang = uni(s, 0.0, 2.0 * kPi);
    sc.dkx[t] = (float)(fx * std::cos(ang) / width);
    sc.dky[t] = (float)(fy * std::sin(ang) / height);
    sc.dp[t] = (float)uni(s, 0.0, 1.0);
    const double a = uni(s, 0.5, 1.0);
    sc.da[t] = (float)a;
    dsum += a;
  }
  sc.dnorm = (float)(1.0 / dsum);
  for (int c = 0; c < 3; ++c) {
    sc.gain[c] = (float)uni(s, 0.9, 1.1);
    sc.offset[c] = (float)uni(s, -10.0, 10.0);
  }
  sc.blur_scale = (float)cfg.blur_scale;
  sc.blur_cap = (float)cfg.blur_cap;
  sc.z = frame_count > 1 ? (float)frame / (float)(frame_count - 1) : 0.5f;
  sc.seed_lo = (uint32_t)seed;
  sc.seed_hi = (uint32_t)(seed >> 32) ^ 0xA5A5A5A5u;
  sc.frame = frame;
  return sc;
}

uint32_t hash3(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u ^ (c + 0x165667B1u) * 0xC2B2AE3Du;
  h ^= h >> 16;
  h *= 0x7FEB352Du;
  h ^= h >> 15;
  h *= 0x846CA68Bu;
  h ^= h >> 16;
  return h;
}

void render_row(const Scene& sc, const or_pose& pose, uint32_t w, uint32_t h, uint32_t y, uint8_t* row) {
  const float twopi = 6.283185307179586f;
  for (uint32_t xs = 0; xs < w; xs += kRun) {
    double X0d, Y0d, X1d, Y1d;
    oracle_forward_point(&pose, w, h, (double)xs, (double)y, &X0d, &Y0d);
    oracle_forward_point(&pose, w, h, (double)(xs + kRun), (double)y, &X1d, &Y1d);
    const float X0 = (float)X0d, Y0 = (float)Y0d;
    const float dX = (float)(X1d - X0d) * (1.0f / kRun), dY = (float)(Y1d - Y0d) * (1.0f / kRun);
    float tex[kRun], att[kRun], rat[kRun];
    for (int j = 0; j < kRun; ++j) {
      const float X = X0 + dX * j, Y = Y0 + dY * j;
      float d = 0.f;
      for (int t = 0; t < kDepthTerms; ++t) {
        const float ph = sc.dkx[t] * X + sc.dky[t] * Y + sc.dp[t];
        d += sc.da[t] * std::cos(twopi * (ph - std::floor(ph)));
      }
      d = 0.5f + 0.5f * d * sc.dnorm;
      const float sigma = std::fmin(std::fabs(d - sc.z) * sc.blur_scale, sc.blur_cap);
      const float s2 = sigma * sigma;
      att[j] = std::exp(-0.5f * s2 * sc.w2_0);
      rat[j] = std::exp(-0.5f * s2 * sc.dw2);
      tex[j] = 0.f;
    }
    for (int i = 0; i < kComp; ++i) {
      const float ph = sc.kx[i] * X0 + sc.ky[i] * Y0 + sc.p0[i];
      float s = std::sin(twopi * (ph - std::floor(ph))), c = std::cos(twopi * (ph - std::floor(ph)));
      const float dph = sc.kx[i] * dX + sc.ky[i] * dY;
      const float sd = std::sin(twopi * dph), cd = std::cos(twopi * dph);
      const float A = sc.amp[i];
      for (int j = 0; j < kRun; ++j) {
        tex[j] += A * att[j] * s;
        att[j] *= rat[j];
        const float ns = s * cd + c * sd;
        c = c * cd - s * sd;
        s = ns;
      }
    }
    for (int j = 0; j < kRun; ++j) {
      const uint32_t x = xs + (uint32_t)j;
      if (x >= w) break;
      uint8_t* o = row + (size_t)x * 3;
      for (int ch = 0; ch < 3; ch += 2) {
        const uint32_t h1 = hash3(sc.seed_lo ^ (sc.frame * 0x632BE5ABu), x * 4u + (uint32_t)ch, y ^ sc.seed_hi);
        const uint32_t h2 = hash3(h1, sc.seed_hi + 0x51ED270Bu, y * 3u + (uint32_t)ch);
        const float u1 = ((h1 >> 8) + 1.0f) * (1.0f / 16777217.0f), u2 = (h2 >> 8) * (1.0f / 16777216.0f);
        const float r = std::sqrt(-2.0f * std::log(u1));
        const float n0 = 4.0f * r * std::cos(twopi * u2), n1 = 4.0f * r * std::sin(twopi * u2);
        for (int e = 0; e < 2 && ch + e < 3; ++e) {
          const int cch = ch + e;
          float v = 128.0f + sc.offset[cch] + sc.gain[cch] * kContrastGain * tex[j] + (e == 0 ? n0 : n1);
          v = std::fmin(std::fmax(std::rint(v), 0.0f), 255.0f);
          o[cch] = (uint8_t)v;
        }
      }
    }
  }
}

}  // namespace

extern "C" {

// Pose of synthetic frame `frame` (the device generator's draws).
void oracle_synth_pose(uint64_t seed, int scene, uint32_t width, uint32_t height, uint32_t frame,
                       uint32_t frame_count, or_pose* out) {
  (void)height;
  (void)frame_count;
  make_pose(seed, scene, width, frame, out);
}

// Render rows [row0, row0 + rows) of synthetic frame `frame` into `out`
// (the whole frame's buffer, interleaved RGB u8, row stride `stride` bytes);
// other rows are left as they are.  Rows are split over `jobs` threads.
void oracle_synth_render(uint64_t seed, int scene, uint32_t width, uint32_t height, uint32_t frame,
                         uint32_t frame_count, uint32_t row0, uint32_t rows, uint8_t* out, size_t stride, int jobs) {
  or_pose pose;
  make_pose(seed, scene, width, frame, &pose);
  const Scene sc = make_scene(seed, scene, width, height, frame, frame_count);
  const uint32_t r1 = row0 + rows > height ? height : row0 + rows;
  if (r1 <= row0) return;
  const uint32_t n = r1 - row0;
  const int nt = jobs < 1 ? 1 : (jobs > (int)n ? (int)n : jobs);
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) {
    th.emplace_back([&, t] {
      for (uint32_t y = row0 + (uint32_t)t; y < r1; y += (uint32_t)nt) render_row(sc, pose, width, height, y, out + (size_t)y * stride);
    });
  }
  for (auto& x : th) x.join();
}

}  // extern "C"
