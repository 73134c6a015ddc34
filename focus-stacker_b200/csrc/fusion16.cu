// 16-bit samples: the remap of u16 frames with support alpha, their
// local-contrast weights, and the level-0 planes pass 2 blends.
//
// The reference keeps u16 twins of the 8-bit path: samplePixelBilinearU16 and
// the soft edge (src/remap.zig:280-336, 443-541, 841-937), gray =
// f32(R + G + B) / (3 * 65535) (src/fuse/grayscale.zig:40-57), the alpha
// weight f32(alpha) / 65535 (src/fuse/masks.zig:6-30) and the quantisation
// to 65535 (src/fuse/pyramid.zig:262-266).  Everything above level 0 is the
// same FP32 pyramid as for 8-bit frames, so a 16-bit stack runs the shared
// level kernels from level 0 on: these kernels produce its level-0 Gaussian
// (the remapped frame as FP32 planes), support and normalised mask.
//
// Every sample takes the exact path: the reference's f64 sampler op for op
// (products and sums rounded one at a time, no fused multiply-add).  An FP32
// fast path would need a rounding-tie band 256 times narrower than the 8-bit
// one.  The contrast statistic sums the reference's f32 gray values in FP64
// over the window, as sampleStdDev expects them (src/fuse/contrast.zig:
// 284-290).
#include <cuda_runtime.h>

#include <cstdint>

#include "fusion_kernels.cuh"

namespace fs {

namespace {

constexpr int TW = kTileW, TH = kTileH, NT = kThreads;
constexpr int PPT = TW * TH / NT;

__device__ __forceinline__ void load_rgb16(const SrcImage& s, int x, int y, double v[3]) {
  const uint16_t* p = reinterpret_cast<const uint16_t*>(s.px + (int64_t)y * s.pitch) + (int64_t)x * s.ch;
  if (s.ch >= 3) {
    v[0] = (double)__ldg(p);
    v[1] = (double)__ldg(p + 1);
    v[2] = (double)__ldg(p + 2);
  } else {
    v[0] = v[1] = v[2] = (double)__ldg(p);
  }
}

__device__ __forceinline__ uint32_t round_u16(double q) { return (uint32_t)fmin(fmax(round(q), 0.0), 65535.0); }

}  // namespace

// Exact u16 sample of output pixel (X, Y): R | G << 16 in .x, B | A << 16
// in .y (samplePixelBilinearU16, src/remap.zig:841-937).
static __device__ uint2 sample_exact16(const Warp& w, const SrcImage& s, int X, int Y) {
  double dx, dy;
  const double Xd = (double)X, Yd = (double)Y;
  const double dD = fma(w.g, Xd, w.h * Yd);
  const double D = dD + 1.0;
  if (w.behind_is_void) {
    if (!(D > 0.0)) return make_uint2(0u, 0u);
  } else if (fabs(D) < w.eps_den) {
    return make_uint2(0u, 0u);
  }
  {
    const double nx = fma(w.a, Xd, fma(w.b, Yd, w.c)) - dD * Xd;
    const double ny = fma(w.d, Xd, fma(w.e, Yd, w.f)) - dD * Yd;
    const double rD = 1.0 / D;
    dx = nx * rD;
    dy = ny * rD;
  }
  int x0, y0;
  double fx, fy;
  if (w.kind == WARP_RADIAL) {
    double ux, uy;
    radial_inverse(w, __dsub_rn(dx + Xd, w.src_cx), __dsub_rn(dy + Yd, w.src_cy), &ux, &uy);
    const double sx = __dadd_rn(w.src_cx, ux), sy = __dadd_rn(w.src_cy, uy);
    const double flx = floor(sx), fly = floor(sy);
    if (!(fabs(flx) < 1e8 && fabs(fly) < 1e8)) return make_uint2(0u, 0u);
    x0 = (int)flx;
    y0 = (int)fly;
    fx = sx - flx;
    fy = sy - fly;
  } else {
    const double flx = floor(dx), fly = floor(dy);
    if (!(fabs(flx) < 1e8 && fabs(fly) < 1e8)) return make_uint2(0u, 0u);
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
  if (!(support > 0.0)) return make_uint2(0u, 0u);
  double val[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (!inb[i]) continue;
    double v[3];
    load_rgb16(s, tx[i], ty[i], v);
#pragma unroll
    for (int c = 0; c < 3; ++c) val[c] = __dadd_rn(val[c], __dmul_rn(v[c], wt[i]));
  }
  uint32_t out[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) out[c] = round_u16(__ddiv_rn(val[c], support));
  const uint32_t alpha = all_in ? 65535u : round_u16(__dmul_rn(support, 65535.0));
  return make_uint2(out[0] | (out[1] << 16), out[2] | (alpha << 16));
}

namespace {

// Pixel (X, Y) of an aligned u16 frame (RGB, alpha 65535, or RGBA).
__device__ __forceinline__ uint2 load_aligned16(const SrcImage& s, int X, int Y) {
  const uint16_t* p = reinterpret_cast<const uint16_t*>(s.px + (int64_t)Y * s.pitch) + (int64_t)X * s.ch;
  const uint32_t al = s.ch == 4 ? (uint32_t)__ldg(p + 3) : 65535u;
  return make_uint2((uint32_t)__ldg(p) | ((uint32_t)__ldg(p + 1) << 16), (uint32_t)__ldg(p + 2) | (al << 16));
}

}  // namespace

// Pass 1 (accumulate: weight sum and union, in frame order) or pass 2
// (planes: level-0 Gaussian, support and normalised mask of each frame) for
// a batch of u16 frames, one 64 x 32 tile per CTA.
template <int B>
__global__ void __launch_bounds__(NT) remap16_weights_kernel(const __grid_constant__ Remap16Args a) {
  constexpr int RW = TW + 2 * B, RH = TH + 2 * B;
  __shared__ uint2 reg[RH * RW];
  __shared__ float gry[RH * RW];  // gray of supported samples, -1 elsewhere
  const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  const int vc = threadIdx.x % TW, vr0 = (threadIdx.x / TW) * PPT;
  const int X = x0 + vc;
  float nacc[PPT];
  uint32_t umask = 0;
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    const int Y = y0 + vr0 + i;
    nacc[i] = 0.0f;
    if (a.accumulate && !a.first && X < a.W && Y < a.H) {
      nacc[i] = a.norm[(int64_t)Y * a.pitch + X];
      if (a.uni[(int64_t)Y * a.pitch + X]) umask |= 1u << i;
    }
  }
  for (int k = 0; k < a.K; ++k) {
    const FrameIn& f = a.f[k];
    for (int i = threadIdx.x; i < RW * RH; i += NT) {
      const int ry = i / RW, rx = i - ry * RW;
      const int Xr = x0 - B + rx, Yr = y0 - B + ry;
      uint2 v = make_uint2(0u, 0u);
      if (Xr >= 0 && Yr >= 0 && Xr < a.W && Yr < a.H)
        v = f.warp.kind == WARP_ALIGNED ? load_aligned16(f.src, Xr, Yr) : sample_exact16(f.warp, f.src, Xr, Yr);
      reg[i] = v;
      const uint32_t k3 = (v.x & 0xFFFFu) + (v.x >> 16) + (v.y & 0xFFFFu);
      gry[i] = (v.y >> 16) > 0 ? __fdiv_rn((float)k3, 196605.0f) : -1.0f;
    }
    __syncthreads();
    const LevelPlanes& out = a.out[k];
#pragma unroll 1
    for (int i = 0; i < PPT; ++i) {
      const int Y = y0 + vr0 + i;
      if (X >= a.W || Y >= a.H) continue;
      const uint2 own = reg[(vr0 + i + B) * RW + vc + B];
      const uint32_t al = own.y >> 16;
      float w = 0.0f;
      if (a.window_ok && al > 0 && X >= B && Y >= B && X < a.W - B && Y < a.H - B) {
        double s = 0.0, ss = 0.0;
        int n = 0;
        for (int dy = 0; dy <= 2 * B; ++dy) {
          const float* row = gry + (vr0 + i + dy) * RW + vc;
#pragma unroll
          for (int dx = 0; dx <= 2 * B; ++dx) {
            const float g = row[dx];
            if (g >= 0.0f) {
              const double gd = (double)g;
              s = __dadd_rn(s, gd);
              ss = __dadd_rn(ss, __dmul_rn(gd, gd));
              ++n;
            }
          }
        }
        float sd = 0.0f;
        if (n > 1) {
          const double var = fmax(__ddiv_rn(__dsub_rn(ss, __ddiv_rn(__dmul_rn(s, s), (double)n)), (double)(n - 1)), 0.0);
          sd = (float)__dsqrt_rn(var);
        }
        w = __fmul_rn(sd, al == 65535u ? 1.0f : __fdiv_rn((float)al, 65535.0f));
      }
      const int64_t o = (int64_t)Y * a.pitch + X;
      if (a.accumulate) {
        nacc[i] = __fadd_rn(nacc[i], w);
        if (al > 0) umask |= 1u << i;
      }
      if (out.g) {
        float* g = (float*)out.g;
        g[o] = (float)(own.x & 0xFFFFu);
        g[out.plane + o] = (float)(own.x >> 16);
        g[2 * out.plane + o] = (float)(own.y & 0xFFFFu);
        out.s[o] = al > 0 ? 1 : 0;
        const float nv = a.norm[o];
        ((float*)out.m)[o] = nv > 1e-12f ? __fdiv_rn(w, nv) : a.inv_count;
      }
    }
    __syncthreads();
  }
  if (a.accumulate) {
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      const int Y = y0 + vr0 + i;
      if (X < a.W && Y < a.H) {
        a.norm[(int64_t)Y * a.pitch + X] = nacc[i];
        a.uni[(int64_t)Y * a.pitch + X] = (uint8_t)((umask >> i) & 1u);
      }
    }
  }
}

cudaError_t launch_remap16_weights(const Remap16Args& a, int border, cudaStream_t s) {
  if (a.K < 1 || a.K > kMaxBatch) return cudaErrorInvalidValue;
  const dim3 grid((a.W + TW - 1) / TW, (a.H + TH - 1) / TH);
  switch (border) {
    case 1: remap16_weights_kernel<1><<<grid, NT, 0, s>>>(a); break;
    case 2: remap16_weights_kernel<2><<<grid, NT, 0, s>>>(a); break;
    case 3: remap16_weights_kernel<3><<<grid, NT, 0, s>>>(a); break;
    case 4: remap16_weights_kernel<4><<<grid, NT, 0, s>>>(a); break;
    case 5: remap16_weights_kernel<5><<<grid, NT, 0, s>>>(a); break;
    case 6: remap16_weights_kernel<6><<<grid, NT, 0, s>>>(a); break;
    case 7: remap16_weights_kernel<7><<<grid, NT, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// Standalone u16 remap (remapU16, src/remap.zig:280-336): ROI-sized output
// with channels + 1 u16 samples per pixel, one pixel per thread.
__global__ void remap16_kernel(const __grid_constant__ RemapArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)a.W * a.H) return;
  const int X = (int)(i % a.W), Y = (int)(i / a.W);
  const uint2 v = sample_exact16(a.f.warp, a.f.src, X, Y);
  uint16_t* d = reinterpret_cast<uint16_t*>(a.dst + (int64_t)Y * a.dst_pitch) + (int64_t)X * a.dst_ch;
  if (a.dst_ch == 4) {
    d[0] = (uint16_t)(v.x & 0xFFFFu);
    d[1] = (uint16_t)(v.x >> 16);
    d[2] = (uint16_t)(v.y & 0xFFFFu);
    d[3] = (uint16_t)(v.y >> 16);
  } else {
    d[0] = (uint16_t)(v.x & 0xFFFFu);
    d[1] = (uint16_t)(v.y >> 16);
  }
}

cudaError_t launch_remap16(const RemapArgs& a, cudaStream_t s) {
  const int64_t n = (int64_t)a.W * a.H;
  remap16_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}

// The blend of a single-level (1 x 1) stack for a batch of frames: acc +=
// G0_k * m_k in frame order (the top level is level 0,
// src/fuse/pyramid.zig:1605-1649).
__global__ void blend_single_level_kernel(float* acc, int64_t acc_plane, const __grid_constant__ Remap16Args a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < a.K; ++k) {
    const float* g = (const float*)a.out[k].g;
    const float m = ((const float*)a.out[k].m)[0];
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c * acc_plane] = __fadd_rn(acc[c * acc_plane], __fmul_rn(g[c * a.out[k].plane], m));
  }
}

cudaError_t launch_blend_single_level(float* acc, int64_t acc_plane, const Remap16Args& a, cudaStream_t s) {
  blend_single_level_kernel<<<1, 32, 0, s>>>(acc, acc_plane, a);
  return cudaGetLastError();
}

}  // namespace fs
