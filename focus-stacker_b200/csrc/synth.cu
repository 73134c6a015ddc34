// Seeded synthetic focus stacks rendered on the device.
//
// Scene (aligned-frame coordinates X, Y):
//   T(X, Y; sigma) = sum_i A_i exp(-sigma^2 w_i^2 / 2) sin(w_i (X cos t_i + Y sin t_i) + p_i)
// with 64 components: amplitudes A_i ~ U(5, 30), orientations t_i ~ U(0, pi),
// phases p_i ~ U(0, 2 pi) and spatial frequencies w_i in [0.05, 1.2] rad/px.
// The w_i^2 lie on an even grid (randomly paired with the other parameters),
// so the Gaussian-blur attenuation exp(-sigma^2 w_i^2 / 2) of consecutive
// components differs by one constant factor per pixel.  The sum is scaled by
// kContrastGain so that its spread (about +-4 sigma = +-120 levels around mid
// grey) stays inside 8 bits; unscaled, 64 such sinusoids would saturate most
// of the frame and create flat clipped windows.
// Depth d(X, Y) in [0, 1]: normalised sum of 6 low-frequency cosines over the
// frame.  Frame k focuses at z_k = k / (F - 1); its blur is
// sigma_k = min(|d - z_k| * s, cap) (s = cap = 3 for the small scene, 8 for
// the production scene).  Per-channel gain / offset, then N(0, 4^2) noise
// (Box-Muller on a counter hash), round and clamp to u8.
// Frame k is rendered on its own pixel grid: source pixel (x, y) shows the
// scene at the forward map of its pose, so remapping with that pose
// realigns it.  Poses: frame 0 identity; others roll U(-r, r) deg, yaw and
// pitch atan(shift / f) with shift U(-s, s) px, focal ratio 1 + U(-0.005, 0.005).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "../../include/focuscuda.h"
#include "fs_host.h"

namespace fs {

namespace {

constexpr int kComp = 64;
constexpr int kDepthTerms = 6;
constexpr float kContrastGain = 0.28f;
constexpr int kRun = 16;  // source pixels per thread along a row

struct Scene {
  float kx[kComp], ky[kComp], p0[kComp], amp[kComp];  // phase in cycles = kx X + ky Y + p0
  float w2_0, dw2;
  float dkx[kDepthTerms], dky[kDepthTerms], dp[kDepthTerms], da[kDepthTerms];
  float dnorm;
  float gain[3], offset[3];
  float blur_scale, blur_cap;
  float z;              // focus plane of the frame
  float fwd[9];         // source pixel -> scene point (row-major homography)
  uint32_t seed_lo, seed_hi, frame;
};

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uni(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }
double uni(uint64_t& s, double lo, double hi) { return lo + (hi - lo) * uni(s); }

const double kPi = 3.14159265358979323846;

__device__ __forceinline__ uint32_t hash3(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u ^ (c + 0x165667B1u) * 0xC2B2AE3Du;
  h ^= h >> 16;
  h *= 0x7FEB352Du;
  h ^= h >> 15;
  h *= 0x846CA68Bu;
  h ^= h >> 16;
  return h;
}

__global__ void synth_kernel(const __grid_constant__ Scene sc, int w, int h, uint8_t* out, int64_t pitch) {
  const int runs_per_row = (w + kRun - 1) / kRun;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= runs_per_row * h) return;
  const int y = id / runs_per_row, xs = (id % runs_per_row) * kRun;
  const float* F = sc.fwd;
  auto map = [&](float x, float& X, float& Y) {
    float nx = F[0] * x + F[1] * y + F[2], ny = F[3] * x + F[4] * y + F[5], d = F[6] * x + F[7] * y + F[8];
    X = nx / d;
    Y = ny / d;
  };
  float X0, Y0, X1, Y1;
  map((float)xs, X0, Y0);
  map((float)(xs + kRun), X1, Y1);
  const float dX = (X1 - X0) * (1.0f / kRun), dY = (Y1 - Y0) * (1.0f / kRun);
  float tex[kRun], att[kRun], rat[kRun];
  const float twopi = 6.283185307179586f;
#pragma unroll
  for (int j = 0; j < kRun; ++j) {
    float X = X0 + dX * j, Y = Y0 + dY * j;
    float d = 0.f;
    for (int t = 0; t < kDepthTerms; ++t) {
      float ph = sc.dkx[t] * X + sc.dky[t] * Y + sc.dp[t];
      d += sc.da[t] * __cosf(twopi * (ph - floorf(ph)));
    }
    d = 0.5f + 0.5f * d * sc.dnorm;
    float sigma = fminf(fabsf(d - sc.z) * sc.blur_scale, sc.blur_cap);
    float s2 = sigma * sigma;
    att[j] = __expf(-0.5f * s2 * sc.w2_0);
    rat[j] = __expf(-0.5f * s2 * sc.dw2);
    tex[j] = 0.f;
  }
  for (int i = 0; i < kComp; ++i) {
    float ph = sc.kx[i] * X0 + sc.ky[i] * Y0 + sc.p0[i];
    float s, c, sd, cd;
    __sincosf(twopi * (ph - floorf(ph)), &s, &c);
    float dph = sc.kx[i] * dX + sc.ky[i] * dY;
    __sincosf(twopi * dph, &sd, &cd);
    const float A = sc.amp[i];
#pragma unroll
    for (int j = 0; j < kRun; ++j) {
      tex[j] = fmaf(A * att[j], s, tex[j]);
      att[j] *= rat[j];
      float ns = s * cd + c * sd;
      c = c * cd - s * sd;
      s = ns;
    }
  }
  for (int j = 0; j < kRun; ++j) {
    int x = xs + j;
    if (x >= w) break;
    uint8_t* o = out + (int64_t)y * pitch + (int64_t)x * 3;
    for (int ch = 0; ch < 3; ch += 2) {
      uint32_t h1 = hash3(sc.seed_lo ^ (sc.frame * 0x632BE5ABu), (uint32_t)x * 4u + ch, (uint32_t)y ^ sc.seed_hi);
      uint32_t h2 = hash3(h1, sc.seed_hi + 0x51ED270Bu, (uint32_t)y * 3u + ch);
      float u1 = ((h1 >> 8) + 1.0f) * (1.0f / 16777217.0f), u2 = (h2 >> 8) * (1.0f / 16777216.0f);
      float r = sqrtf(-2.0f * __logf(u1));
      float ss, cc;
      __sincosf(twopi * u2, &ss, &cc);
      float n0 = 4.0f * r * cc, n1 = 4.0f * r * ss;
      for (int e = 0; e < 2 && ch + e < 3; ++e) {
        int cch = ch + e;
        float v = 128.0f + sc.offset[cch] + sc.gain[cch] * kContrastGain * tex[j] + (e == 0 ? n0 : n1);
        v = fminf(fmaxf(rintf(v), 0.0f), 255.0f);
        o[cch] = (uint8_t)v;
      }
    }
  }
}

struct SceneConfig {
  double blur_scale, blur_cap, shift, roll_deg;
};
SceneConfig scene_config(int scene) {
  if (scene == 0) return {3.0, 3.0, 20.0, 0.2};
  return {8.0, 8.0, 60.0, 0.3};
}

double focal_px(uint32_t width, double hfov_deg) { return ((double)width * 0.5) / std::tan(hfov_deg * kPi / 360.0); }

bool invert3(const double m[9], double r[9]) {
  double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
  if (!(std::fabs(det) > 0)) return false;
  double id = 1.0 / det;
  r[0] = (m[4] * m[8] - m[5] * m[7]) * id;
  r[1] = (m[2] * m[7] - m[1] * m[8]) * id;
  r[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  r[3] = (m[5] * m[6] - m[3] * m[8]) * id;
  r[4] = (m[0] * m[8] - m[2] * m[6]) * id;
  r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  r[6] = (m[3] * m[7] - m[4] * m[6]) * id;
  r[7] = (m[1] * m[6] - m[0] * m[7]) * id;
  r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
  return true;
}

}  // namespace

void synth_pose(uint64_t seed, int scene, uint32_t width, uint32_t height, uint32_t frame, uint32_t frame_count,
                fs_pose* p) {
  (void)height;
  (void)frame_count;
  fs_pose_default(p);
  if (frame == 0) return;
  SceneConfig cfg = scene_config(scene);
  uint64_t s = seed * 0x2545F4914F6CDD1Dull + 0x1000ull * (frame + 1);
  double f = focal_px(width, p->base_hfov_degrees);
  double sx = uni(s, -cfg.shift, cfg.shift), sy = uni(s, -cfg.shift, cfg.shift);
  p->roll = uni(s, -cfg.roll_deg, cfg.roll_deg) * kPi / 180.0;
  p->yaw = std::atan(sx / f);
  p->pitch = std::atan(sy / f);
  double ratio = 1.0 + uni(s, -0.005, 0.005);
  double hfov = 2.0 * std::atan((double)width * 0.5 / (f * ratio)) * 180.0 / kPi;
  p->hfov_delta = hfov - p->base_hfov_degrees;
}

int synth_render(uint64_t seed, int scene, uint32_t width, uint32_t height, uint32_t frame, uint32_t frame_count,
                 void* dev_out, size_t out_stride, fs_pose* pose_out, cudaStream_t stream, const char** why) {
  fs_pose pose;
  synth_pose(seed, scene, width, height, frame, frame_count, &pose);
  if (pose_out) *pose_out = pose;
  SceneConfig cfg = scene_config(scene);
  Scene sc;
  std::memset(&sc, 0, sizeof(sc));
  uint64_t s = seed * 0x9E3779B97F4A7C15ull + 17;
  const double wmin = 0.05, wmax = 1.2;
  sc.w2_0 = (float)(wmin * wmin);
  sc.dw2 = (float)((wmax * wmax - wmin * wmin) / (kComp - 1));
  int order[kComp];
  for (int i = 0; i < kComp; ++i) order[i] = i;
  for (int i = kComp - 1; i > 0; --i) {
    int j = (int)(splitmix(s) % (uint64_t)(i + 1));
    int t = order[i];
    order[i] = order[j];
    order[j] = t;
  }
  // component i carries frequency grid index i (attenuation recurrence);
  // orientation / phase / amplitude come from the shuffled draw
  double A[kComp], T[kComp], P[kComp];
  for (int i = 0; i < kComp; ++i) {
    A[i] = uni(s, 5.0, 30.0);
    T[i] = uni(s, 0.0, kPi);
    P[i] = uni(s, 0.0, 2.0 * kPi);
  }
  for (int i = 0; i < kComp; ++i) {
    int o = order[i];
    double w = std::sqrt(wmin * wmin + (wmax * wmax - wmin * wmin) * i / (kComp - 1.0));
    sc.kx[i] = (float)(w * std::cos(T[o]) / (2.0 * kPi));
    sc.ky[i] = (float)(w * std::sin(T[o]) / (2.0 * kPi));
    sc.p0[i] = (float)(P[o] / (2.0 * kPi));
    sc.amp[i] = (float)A[o];
  }
  double dsum = 0.0;
  for (int t = 0; t < kDepthTerms; ++t) {
    double fx = uni(s, 0.3, 2.0), fy = uni(s, 0.3, 2.0);
    double ang = uni(s, 0.0, 2.0 * kPi);
    sc.dkx[t] = (float)(fx * std::cos(ang) / width);
    sc.dky[t] = (float)(fy * std::sin(ang) / height);
    sc.dp[t] = (float)uni(s, 0.0, 1.0);
    double a = uni(s, 0.5, 1.0);
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
  // forward map = inverse of the composed output -> source homography
  double Hs[9];
  {
    fs_rect full = {0, 0, (int32_t)width, (int32_t)height};
    Warp w;
    if (!compose_warp(pose, width, height, full, &w, why)) return FS_ERR_INVALID;
    double H[9] = {1 + w.a, w.b, w.c, w.d, 1 + w.e, w.f, w.g, w.h, 1};
    if (!invert3(H, Hs)) {
      if (why) *why = "singular synthetic pose";
      return FS_ERR_INVALID;
    }
  }
  for (int i = 0; i < 9; ++i) sc.fwd[i] = (float)Hs[i];
  int runs = (int)((width + kRun - 1) / kRun) * (int)height;
  synth_kernel<<<(runs + 127) / 128, 128, 0, stream>>>(sc, (int)width, (int)height, (uint8_t*)dev_out,
                                                      (int64_t)out_stride);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    if (why) *why = cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

}  // namespace fs
