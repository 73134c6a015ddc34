// sm_100a kernels of the remap + pyramid-contrast fusion path.
//
// Pass 1  pass1_kernel      remap -> gray -> local contrast -> alpha weight
//                           -> weight sum (frame order) and union support
// Pass 2  level_kernel<0>   remap -> weight -> normalise -> level-0 Gaussian
//                           and mask -> level-1 REDUCE of both -> EXPAND ->
//                           Laplacian x mask into the level-0 accumulator
//         level_kernel<1>   the same step for level l >= 1 from HBM planes
// Final   collapse_kernel   parent += EXPAND(child), quantise at level 0
//
// All of it is HBM-bandwidth bound stencil work on CUDA cores (no tensor
// cores): 64x32 tiles staged in shared memory with their halos, frames of a
// batch (K <= 8) processed inside one CTA so that per-pixel state (weight
// sums, accumulators) is read and written once per batch while the frame
// order of every FP32 sum stays the reference's.
#include <cuda_runtime.h>

#include "fusion_kernels.cuh"

namespace fs {

namespace {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ float kw(int i) { return (i == 0 || i == 4) ? 1.0f : ((i == 1 || i == 3) ? 4.0f : 6.0f); }

// ------------------------------------------------------------ region remap
// Fill a shared region of packed RGBA samples for output pixels
// [rx0, rx0 + rw) x [ry0, ry0 + rh) (ROI coordinates).  Pixels outside the
// ROI get 0 (alpha 0 = no support).  Work unit: 8x4 pixel blocks, one warp
// each, sharing one double-float anchor.
__device__ void fill_region(const FrameIn& f, int W, int H, int rx0, int ry0, int rw, int rh, uint32_t* reg) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  if (f.warp.kind == WARP_ALIGNED) {
    for (int i = threadIdx.x; i < rw * rh; i += blockDim.x) {
      int rx = i % rw, ry = i / rw;
      int X = rx0 + rx, Y = ry0 + ry;
      uint32_t v = 0;
      if (X >= 0 && Y >= 0 && X < W && Y < H) {
        const uint8_t* p = f.src.px + (int64_t)Y * f.src.pitch + (int64_t)X * f.src.ch;
        uint32_t a = f.src.ch == 4 ? (uint32_t)__ldg(p + 3) : 255u;
        v = pack_rgba(__ldg(p), __ldg(p + 1), __ldg(p + 2), a);
      }
      reg[i] = v;
    }
    return;
  }
  const int nbx = (rw + 7) >> 3, nby = (rh + 3) >> 2, nb = nbx * nby;
  const int du = lane & 7, dv = lane >> 3;
  const bool fast_ok = f.warp.kind == WARP_HOMOGRAPHY && !f.warp.guard;
  // this warp handles blocks warp, warp + nwarps, ...; lane j forms the
  // anchor of the j-th of up to 32 of them, then each block takes it by shuffle
  for (int g0 = warp; g0 < nb; g0 += nwarps * 32) {
    Anchor mine = {};
    bool mine_ok = false;
    {
      const int bj = g0 + lane * nwarps;
      if (fast_ok && bj < nb) mine = make_anchor(f.warp, rx0 + (bj % nbx) * 8, ry0 + (bj / nbx) * 4, &mine_ok);
    }
    const int cnt = min(32, (nb - g0 + nwarps - 1) / nwarps);
    for (int j = 0; j < cnt; ++j) {
      const int blk = g0 + j * nwarps;
      const int bx = blk % nbx, by = blk / nbx;
      const int AX = rx0 + bx * 8, AY = ry0 + by * 4;
      const bool aok = __shfl_sync(0xffffffffu, mine_ok ? 1 : 0, j) != 0;
      const Anchor an = shfl_anchor(mine, j);
      const int rx = bx * 8 + du, ry = by * 4 + dv;
      if (rx >= rw || ry >= rh) continue;
      const int X = AX + du, Y = AY + dv;
      uint32_t v = 0;
      if (X >= 0 && Y >= 0 && X < W && Y < H) {
        v = aok ? sample_fast(f.warp, f.src, an, du, dv, X, Y) : sample_exact(f.warp, f.src, X, Y);
      }
      reg[ry * rw + rx] = v;
    }
  }
}

__device__ __forceinline__ uint32_t px_alpha(uint32_t v) { return v >> 24; }
__device__ __forceinline__ int px_gray(uint32_t v) { return (int)(v & 255u) + (int)((v >> 8) & 255u) + (int)((v >> 16) & 255u); }
__device__ __forceinline__ float px_chan(uint32_t v, int c) { return (float)((v >> (8 * c)) & 255u); }

// f32(alpha) / 255 as the reference computes it (src/fuse/masks.zig:18).
__device__ __forceinline__ float alpha_support(uint32_t al) {
  return al == 255u ? 1.0f : __fdiv_rn((float)al, 255.0f);
}

// Sample standard deviation of gray = k / 765 over the supported window
// pixels, from exact integer sums of k and k^2 (src/fuse/contrast.zig:284-290):
// var = (n S2 - S1^2) / (n (n - 1) 765^2).
__device__ __forceinline__ float window_stddev(int n, long long s1, long long s2) {
  if (n <= 1) return 0.0f;
  long long num = (long long)n * s2 - s1 * s1;
  if (num <= 0) return 0.0f;
  float den = (float)((long long)n * (n - 1)) * 585225.0f;
  return sqrtf(__fdividef((float)num, den));
}

}  // namespace

// ================================================================= pass 1
size_t pass1_smem_bytes(int border) {
  int rw = kTileW + 2 * border, rh = kTileH + 2 * border;
  return (size_t)rw * rh * 4 + (size_t)rh * kTileW * (4 + 4 + 4) + 16;
}

__global__ void __launch_bounds__(kThreads) pass1_kernel(const __grid_constant__ Pass1Args a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int b = a.border;
  const int rw = kTileW + 2 * b, rh = kTileH + 2 * b;
  uint32_t* reg = (uint32_t*)smem;
  int* hn = (int*)(reg + rw * rh);
  int* hs1 = hn + rh * kTileW;
  uint32_t* hs2 = (uint32_t*)(hs1 + rh * kTileW);
  const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * kTileH;
  constexpr int PPT = kTileW * kTileH / kThreads;  // output pixels per thread
  float nacc[PPT];
  uint32_t umask = 0;  // union support of this thread's pixels, one bit each
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    int p = threadIdx.x + i * kThreads;
    int X = x0 + (p % kTileW), Y = y0 + (p / kTileW);
    nacc[i] = 0.0f;
    if (!a.first && X < a.W && Y < a.H) {
      nacc[i] = a.norm[(int64_t)Y * a.norm_pitch + X];
      if (a.uni[(int64_t)Y * a.uni_pitch + X]) umask |= 1u << i;
    }
  }
  for (int k = 0; k < a.K; ++k) {
    fill_region(a.f[k], a.W, a.H, x0 - b, y0 - b, rw, rh, reg);
    __syncthreads();
    // horizontal window sums: region row r, output column c -> cols [c, c + 2b]
    for (int i = threadIdx.x; i < rh * kTileW; i += blockDim.x) {
      int r = i / kTileW, c = i % kTileW;
      const uint32_t* row = reg + r * rw + c;
      int n = 0, s1 = 0;
      uint32_t s2 = 0;
      for (int t = 0; t <= 2 * b; ++t) {
        uint32_t v = row[t];
        if (px_alpha(v) > 0) {
          int g = px_gray(v);
          n += 1;
          s1 += g;
          s2 += (uint32_t)(g * g);
        }
      }
      hn[i] = n;
      hs1[i] = s1;
      hs2[i] = s2;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      int p = threadIdx.x + i * kThreads;
      int c = p % kTileW, r = p / kTileW;
      int X = x0 + c, Y = y0 + r;
      if (X >= a.W || Y >= a.H) continue;
      uint32_t own = reg[(r + b) * rw + (c + b)];
      uint32_t al = px_alpha(own);
      if (al > 0) umask |= 1u << i;
      float w = 0.0f;
      if (a.window_ok && al > 0 && X >= b && Y >= b && X < a.W - b && Y < a.H - b) {
        int n = 0;
        long long s1 = 0, s2 = 0;
        for (int t = 0; t <= 2 * b; ++t) {
          int j = (r + t) * kTileW + c;
          n += hn[j];
          s1 += hs1[j];
          s2 += hs2[j];
        }
        float sd = window_stddev(n, s1, s2);
        w = __fmul_rn(sd, alpha_support(al));
      }
      nacc[i] = __fadd_rn(nacc[i], w);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    int p = threadIdx.x + i * kThreads;
    int X = x0 + (p % kTileW), Y = y0 + (p / kTileW);
    if (X < a.W && Y < a.H) {
      a.norm[(int64_t)Y * a.norm_pitch + X] = nacc[i];
      a.uni[(int64_t)Y * a.uni_pitch + X] = (uint8_t)((umask >> i) & 1u);
    }
  }
}

cudaError_t launch_pass1(const Pass1Args& a, cudaStream_t s) {
  size_t sm = pass1_smem_bytes(a.border);
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(pass1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  dim3 grid((a.W + kTileW - 1) / kTileW, (a.H + kTileH - 1) / kTileH);
  pass1_kernel<<<grid, kThreads, sm, s>>>(a);
  return cudaGetLastError();
}

// =========================================================== level kernel
// Shared-memory geometry of one level step (tile origin x0, y0 at level l;
// level-(l+1) tile origin x1 = x0 / 2, y1 = y0 / 2):
//   G region   level-l cols [x0 - 4, x0 + TW + 2], rows [y0 - 4, y0 + TH + 2]
//              (feeds level-(l+1) Gaussians on the tile plus a 1-pixel halo,
//              which the expand back to the tile needs)
//   M region   level-l cols [x0 - 2, x0 + TW], rows [y0 - 2, y0 + TH]
//              (feeds the level-(l+1) mask on the tile)
//   N tile     level-(l+1) cols [x1 - 1, x1 + TW/2], rows [y1 - 1, y1 + TH/2]
namespace {

constexpr int GW = kTileW + 7, GH = kTileH + 7;          // G region
constexpr int MW = kTileW + 3, MH = kTileH + 3;          // M region
constexpr int NW = kTileW / 2 + 2, NH = kTileH / 2 + 2;  // level l+1 tile + halo
constexpr int TW1 = kTileW / 2, TH1 = kTileH / 2;
constexpr int kTmpFloats = (GH * NW * 4 > NH * kTileW * 3) ? GH * NW * 4 : NH * kTileW * 3;
constexpr int kPPT = kTileW * kTileH / kThreads;

struct LevelSmem {
  float ng[3][NH * NW];     // level-(l+1) Gaussian (zero outside the level)
  float nm[TH1 * TW1];      // level-(l+1) mask on the tile
  float m[MH * MW];         // level-l mask (M region)
  float tmp[kTmpFloats];    // reduce / expand temporaries (and level-0 contrast sums)
  uint8_t ns[NH * NW];      // level-(l+1) support
  uint8_t sm[MH * MW];      // level-l mask support (M region)
};

// Horizontal stage of EXPAND for output column x from a child row g[]
// indexed by child column - (cx1 - 1), exactly in the reference's operation
// order.  clamped (parent larger than 512): src/fuse/pyramid.zig:1748-1775,
// even 2j: (s[j-1] + 6 s[j] + s[j+1]) * 1/8, odd 2j+1: (s[j] + s[j+1]) * 1/2
// with clamped coordinates.  no-wrap (parent at most 512):
// src/fuse/pyramid.zig:1167-1354, (s[j-1] + 6 s[j]) + s[j+1] and
// 4 (s[j] + s[j+1]) with zero outside (g holds 0 there); the division by the
// position-dependent normaliser comes after the vertical stage.
__device__ __forceinline__ float expand_h(const float* g, int x, int cx1, int wc, bool exact) {
  const int j = x >> 1, o = cx1 - 1;
  if (!exact) {
    if ((x & 1) == 0) {
      float s0 = g[clampi(j - 1, 0, wc - 1) - o], s1 = g[clampi(j, 0, wc - 1) - o], s2 = g[clampi(j + 1, 0, wc - 1) - o];
      return __fmul_rn(__fadd_rn(__fadd_rn(s0, __fmul_rn(6.0f, s1)), s2), 0.125f);
    }
    float s0 = g[clampi(j, 0, wc - 1) - o], s1 = g[clampi(j + 1, 0, wc - 1) - o];
    return __fmul_rn(__fadd_rn(s0, s1), 0.5f);
  }
  if ((x & 1) == 0) return __fadd_rn(__fadd_rn(g[j - 1 - o], __fmul_rn(6.0f, g[j - o])), g[j + 1 - o]);
  return __fmul_rn(4.0f, __fadd_rn(g[j - o], g[j + 1 - o]));
}

// Vertical stage for output (x, y) from horizontal rows hrow[(row - (cy1 - 1)) * rstride + col] (x channel
// already selected by the caller through `col`).  clamped: even 2i: (r[i-1] + 6 r[i] + r[i+1]) * 1/8,
// odd 2i+1: (r[i] + r[i]) * 1/2 (the reference reads row i twice,
// src/fuse/pyramid.zig:1122-1145); no-wrap: (r[i-1] + 6 r[i]) + r[i+1] or
// r[i] + r[i+1] with zero outside, divided by the normaliser.
__device__ __forceinline__ float expand_v(const float* hrow, int rstride, int col, int x, int y, int cy1, int wc,
                                          int hc, bool exact) {
  const int q = y >> 1, o = cy1 - 1;
  if (!exact) {
    if ((y & 1) == 0) {
      float r0 = hrow[(clampi(q - 1, 0, hc - 1) - o) * rstride + col];
      float r1 = hrow[(clampi(q, 0, hc - 1) - o) * rstride + col];
      float r2 = hrow[(clampi(q + 1, 0, hc - 1) - o) * rstride + col];
      return __fmul_rn(__fadd_rn(__fadd_rn(r0, __fmul_rn(6.0f, r1)), r2), 0.125f);
    }
    float r0 = hrow[(clampi(q, 0, hc - 1) - o) * rstride + col];
    return __fmul_rn(__fadd_rn(r0, r0), 0.5f);
  }
  auto row = [&](int qq) -> float { return (qq < 0 || qq >= hc) ? 0.0f : hrow[(qq - o) * rstride + col]; };
  float v = ((y & 1) == 0) ? __fadd_rn(__fadd_rn(row(q - 1), __fmul_rn(6.0f, row(q))), row(q + 1))
                           : __fadd_rn(row(q), row(q + 1));
  return __fdiv_rn(v, exact_expand_divisor(x, y, wc, hc));
}

template <bool FRAME>
struct GSource;

// Level 0: the G region holds packed RGBA samples of the frame.
template <>
struct GSource<true> {
  const uint32_t* reg;  // G region, row-major GW wide
  __device__ float g(int c, int rx, int ry) const { return px_chan(reg[ry * GW + rx], c); }
  __device__ bool s(int rx, int ry) const { return px_alpha(reg[ry * GW + rx]) > 0; }
};
// Level >= 1: planar FP32 Gaussian and u8 support.
template <>
struct GSource<false> {
  const float* gp;      // 3 planes of GH * GW
  const uint8_t* sp;
  __device__ float g(int c, int rx, int ry) const { return gp[c * GH * GW + ry * GW + rx]; }
  __device__ bool s(int rx, int ry) const { return sp[ry * GW + rx] != 0; }
};

// REDUCE with support to the level-(l+1) tile (+ halo for the Gaussian),
// src/fuse/pyramid.zig:997-1099: 5x5 taps [1 4 6 4 1]^2 over in-range
// samples with support > 0, value = sum(w v) / sum(w), support = sum(w) > 0.
// Evaluated separably (rows first); the weights are exact small integers.
template <bool FRAME>
__device__ void reduce_step(const GSource<FRAME>& src, LevelSmem& S, const LevelArgs& a, int x0, int y0) {
  const int x1 = x0 >> 1, y1 = y0 >> 1;
  float* th = S.tmp;  // [GH][NW][4]
  for (int i = threadIdx.x; i < GH * NW; i += blockDim.x) {
    int ry = i / NW, jj = i % NW;
    int j = x1 - 1 + jj;
    float v0 = 0.f, v1 = 0.f, v2 = 0.f, ws = 0.f;
#pragma unroll
    for (int kx = 0; kx < 5; ++kx) {
      int sx = 2 * j - 2 + kx;
      if (sx < 0 || sx >= a.wl) continue;
      int rx = sx - (x0 - 4);
      if (!src.s(rx, ry)) continue;
      float w = kw(kx);
      v0 = fmaf(w, src.g(0, rx, ry), v0);
      v1 = fmaf(w, src.g(1, rx, ry), v1);
      v2 = fmaf(w, src.g(2, rx, ry), v2);
      ws += w;
    }
    float* o = th + i * 4;
    o[0] = v0; o[1] = v1; o[2] = v2; o[3] = ws;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NH * NW; i += blockDim.x) {
    int ii = i / NW, jj = i % NW;
    int yi = y1 - 1 + ii, xj = x1 - 1 + jj;
    float v0 = 0.f, v1 = 0.f, v2 = 0.f, ws = 0.f;
#pragma unroll
    for (int ky = 0; ky < 5; ++ky) {
      int sy = 2 * yi - 2 + ky;
      if (sy < 0 || sy >= a.hl) continue;
      int ry = sy - (y0 - 4);
      const float* t = th + (ry * NW + jj) * 4;
      float w = kw(ky);
      v0 = fmaf(w, t[0], v0);
      v1 = fmaf(w, t[1], v1);
      v2 = fmaf(w, t[2], v2);
      ws = fmaf(w, t[3], ws);
    }
    bool inside = xj >= 0 && yi >= 0 && xj < a.wn && yi < a.hn;
    bool sup = inside && ws > 0.f;
    S.ng[0][i] = sup ? v0 / ws : 0.f;
    S.ng[1][i] = sup ? v1 / ws : 0.f;
    S.ng[2][i] = sup ? v2 / ws : 0.f;
    S.ns[i] = sup ? 1 : 0;
  }
  __syncthreads();
  float* tm = S.tmp;  // [MH][TW1][2]
  for (int i = threadIdx.x; i < MH * TW1; i += blockDim.x) {
    int ry = i / TW1, jj = i % TW1;
    int j = x1 + jj;
    float v = 0.f, ws = 0.f;
#pragma unroll
    for (int kx = 0; kx < 5; ++kx) {
      int sx = 2 * j - 2 + kx;
      if (sx < 0 || sx >= a.wl) continue;
      int rx = sx - (x0 - 2);
      if (!S.sm[ry * MW + rx]) continue;
      float w = kw(kx);
      v = fmaf(w, S.m[ry * MW + rx], v);
      ws += w;
    }
    tm[i * 2] = v;
    tm[i * 2 + 1] = ws;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < TH1 * TW1; i += blockDim.x) {
    int ii = i / TW1, jj = i % TW1;
    int yi = y1 + ii;
    float v = 0.f, ws = 0.f;
#pragma unroll
    for (int ky = 0; ky < 5; ++ky) {
      int sy = 2 * yi - 2 + ky;
      if (sy < 0 || sy >= a.hl) continue;
      int ry = sy - (y0 - 2);
      float w = kw(ky);
      v = fmaf(w, tm[(ry * TW1 + jj) * 2], v);
      ws = fmaf(w, tm[(ry * TW1 + jj) * 2 + 1], ws);
    }
    S.nm[i] = ws > 0.f ? v / ws : 0.f;
  }
  __syncthreads();
}

// Store the level-(l+1) tile (Gaussian, support, mask) of one frame, or add
// it into the top accumulator when l + 1 is the last level
// (src/fuse/pyramid.zig:1533-1554, 1605-1649).
__device__ void store_next(const LevelSmem& S, const LevelArgs& a, int x0, int y0, int k) {
  const int x1 = x0 >> 1, y1 = y0 >> 1;
  const bool top = a.level + 1 == a.levels - 1;
  for (int i = threadIdx.x; i < TH1 * TW1; i += blockDim.x) {
    int ii = i / TW1, jj = i % TW1;
    int xj = x1 + jj, yi = y1 + ii;
    if (xj >= a.wn || yi >= a.hn) continue;
    int ni = (ii + 1) * NW + (jj + 1);
    int64_t o = (int64_t)yi * a.pitch_n + xj;
    if (top) {
      float m = S.nm[i];
      for (int c = 0; c < 3; ++c) {
        float* acc = a.acc_n + c * a.acc_plane_n + o;
        *acc = __fadd_rn(*acc, __fmul_rn(S.ng[c][ni], m));
      }
    } else {
      const LevelPlanes& out = a.out[k];
      for (int c = 0; c < 3; ++c) out.g[c * out.plane + o] = S.ng[c][ni];
      out.s[o] = S.ns[ni];
      out.m[o] = S.nm[i];
    }
  }
}

// EXPAND of the level-(l+1) Gaussian back to the level-l tile fused with the
// weighted Laplacian blend into the accumulator registers:
// acc += (G_l - EXPAND(G_{l+1})) * M_l  (src/fuse/pyramid.zig:1480-1504).
template <bool FRAME>
__device__ void expand_blend_step(const GSource<FRAME>& src, LevelSmem& S, const LevelArgs& a, int x0, int y0,
                                  float (&acc)[kPPT][3]) {
  const int x1 = x0 >> 1, y1 = y0 >> 1;
  float* hrow = S.tmp;  // [NH][TW][3]
  const bool exact = a.exact_expand != 0;
  for (int i = threadIdx.x; i < NH * kTileW; i += blockDim.x) {
    int ii = i / kTileW, xx = i % kTileW;
    int yi = y1 - 1 + ii;
    if (yi < 0 || yi >= a.hn) continue;
    for (int c = 0; c < 3; ++c) hrow[i * 3 + c] = expand_h(S.ng[c] + ii * NW, x0 + xx, x1, a.wn, exact);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kPPT; ++i) {
    int p = threadIdx.x + i * kThreads;
    int xx = p % kTileW, yy = p / kTileW;
    int x = x0 + xx, y = y0 + yy;
    if (x >= a.wl || y >= a.hl) continue;
    float m = S.m[(yy + 2) * MW + (xx + 2)];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float e = expand_v(hrow, kTileW * 3, xx * 3 + c, x, y, y1, a.wn, a.hn, exact);
      float lap = __fsub_rn(src.g(c, xx + 4, yy + 4), e);
      acc[i][c] = __fadd_rn(acc[i][c], __fmul_rn(lap, m));
    }
  }
  __syncthreads();
}

struct ContrastSums {
  uint8_t* n;
  uint16_t* s1;
  uint32_t* s2;
};

__host__ __device__ constexpr size_t contrast_bytes(int border) {
  return (size_t)(kTileH + 3 + 2 * border) * MW * (1 + 2 + 4) + 32;
}

}  // namespace

size_t level_smem_bytes() { return sizeof(LevelSmem) + 16 + (size_t)3 * GH * GW * 4 + (size_t)GH * GW; }
size_t level0_smem_bytes(int border) {
  int hb = border > 2 ? border : 2;
  size_t rw = kTileW + 2 * hb + 3, rh = kTileH + 2 * hb + 3;
  size_t bytes = sizeof(LevelSmem) + 16 + rw * rh * 4 + (size_t)MH * MW * 4;
  if (contrast_bytes(border) > sizeof(float) * kTmpFloats) bytes += contrast_bytes(border);
  return bytes;
}

// Level step l -> l + 1 for a batch of frames.  FRAME: level 0, built from
// the input frame (remap + weights); otherwise level l >= 1 from HBM.
template <bool FRAME>
__global__ void __launch_bounds__(kThreads) level_kernel(const __grid_constant__ LevelArgs a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  LevelSmem& S = *reinterpret_cast<LevelSmem*>(smem_raw);
  uint8_t* extra = smem_raw + ((sizeof(LevelSmem) + 15) & ~(size_t)15);
  const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * kTileH;
  const int b = a.border;
  const int hb = b > 2 ? b : 2;
  float* normr = nullptr;
  uint32_t* reg = nullptr;
  int rw = 0, rh = 0;
  ContrastSums cs = {nullptr, nullptr, nullptr};
  float* gpl = nullptr;
  uint8_t* spl = nullptr;
  const int crh = kTileH + 3 + 2 * b;  // contrast rows [y0 - 2 - b, y0 + TH + b]
  if (FRAME) {
    rw = kTileW + 2 * hb + 3;
    rh = kTileH + 2 * hb + 3;
    reg = (uint32_t*)extra;
    normr = (float*)(reg + rw * rh);
    uint8_t* cbase = contrast_bytes(b) > sizeof(float) * kTmpFloats ? (uint8_t*)(normr + MH * MW) : (uint8_t*)S.tmp;
    cs.s2 = (uint32_t*)cbase;
    cs.s1 = (uint16_t*)(cs.s2 + crh * MW);
    cs.n = (uint8_t*)(cs.s1 + crh * MW);
  } else {
    gpl = (float*)extra;
    spl = (uint8_t*)(gpl + 3 * GH * GW);
  }
  // frame-independent inputs: mask support (and at level 0 the weight sums)
  for (int i = threadIdx.x; i < MH * MW; i += blockDim.x) {
    int X = x0 - 2 + i % MW, Y = y0 - 2 + i / MW;
    bool in = X >= 0 && Y >= 0 && X < a.wl && Y < a.hl;
    int64_t o = (int64_t)Y * a.pitch_l + X;
    S.sm[i] = in ? a.sm_l[o] : 0;
    if (FRAME) normr[i] = in ? a.norm[o] : 0.0f;
  }
  float acc[kPPT][3];
#pragma unroll
  for (int i = 0; i < kPPT; ++i) {
    int p = threadIdx.x + i * kThreads;
    int X = x0 + p % kTileW, Y = y0 + p / kTileW;
    bool in = X < a.wl && Y < a.hl;
    int64_t o = (int64_t)Y * a.pitch_l + X;
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[i][c] = in ? a.acc_l[c * a.acc_plane_l + o] : 0.0f;
  }
  __syncthreads();
  for (int k = 0; k < a.K; ++k) {
    if (FRAME) {
      // ---- remap the frame over the G region plus the contrast halo
      const int rx0 = x0 - 2 - hb, ry0 = y0 - 2 - hb;
      fill_region(a.f[k], a.wl, a.hl, rx0, ry0, rw, rh, reg);
      __syncthreads();
      // ---- local contrast over the M region (src/fuse/contrast.zig:96-282)
      for (int i = threadIdx.x; i < crh * MW; i += blockDim.x) {
        int r = i / MW, c = i % MW;
        int ry = (y0 - 2 - b + r) - ry0, rx = (x0 - 2 + c - b) - rx0;
        const uint32_t* row = reg + ry * rw + rx;
        int n = 0, s1 = 0;
        uint32_t s2 = 0;
        for (int t = 0; t <= 2 * b; ++t) {
          uint32_t v = row[t];
          if (px_alpha(v) > 0) {
            int g = px_gray(v);
            n += 1;
            s1 += g;
            s2 += (uint32_t)(g * g);
          }
        }
        cs.n[i] = (uint8_t)n;
        cs.s1[i] = (uint16_t)s1;
        cs.s2[i] = s2;
      }
      __syncthreads();
      // ---- weight, alpha, normalise -> level-0 mask (src/fuse/pyramid.zig:303-316)
      for (int i = threadIdx.x; i < MH * MW; i += blockDim.x) {
        int c = i % MW, r = i / MW;
        int X = x0 - 2 + c, Y = y0 - 2 + r;
        float mval = 0.0f;
        if (X >= 0 && Y >= 0 && X < a.wl && Y < a.hl) {
          uint32_t own = reg[(Y - ry0) * rw + (X - rx0)];
          uint32_t al = px_alpha(own);
          float w = 0.0f;
          if (a.window_ok && al > 0 && X >= b && Y >= b && X < a.wl - b && Y < a.hl - b) {
            int n = 0;
            long long s1 = 0, s2 = 0;
            for (int t = 0; t <= 2 * b; ++t) {
              int j = (r + t) * MW + c;
              n += cs.n[j];
              s1 += cs.s1[j];
              s2 += cs.s2[j];
            }
            w = __fmul_rn(window_stddev(n, s1, s2), alpha_support(al));
          }
          float nv = normr[i];
          mval = nv > 1e-12f ? __fdiv_rn(w, nv) : a.inv_count;
        }
        S.m[i] = mval;
      }
      __syncthreads();
      GSource<true> src;
      src.reg = reg;
      if (rw != GW || hb != 2) {
        // border > 2: compact the G region out of the wider remap region
        uint32_t* comp = (uint32_t*)S.tmp;
        for (int i = threadIdx.x; i < GH * GW; i += blockDim.x)
          comp[i] = reg[(i / GW + hb - 2) * rw + (i % GW + hb - 2)];
        __syncthreads();
        for (int i = threadIdx.x; i < GH * GW; i += blockDim.x) reg[i] = comp[i];
        __syncthreads();
      }
      if (a.levels == 1) {
        // 1x1 image: the top level is level 0 (src/fuse/pyramid.zig:1605-1649)
#pragma unroll
        for (int i = 0; i < kPPT; ++i) {
          int p = threadIdx.x + i * kThreads;
          int xx = p % kTileW, yy = p / kTileW;
          if (x0 + xx >= a.wl || y0 + yy >= a.hl) continue;
          float m = S.m[(yy + 2) * MW + (xx + 2)];
          for (int c = 0; c < 3; ++c) acc[i][c] = __fadd_rn(acc[i][c], __fmul_rn(src.g(c, xx + 4, yy + 4), m));
        }
        __syncthreads();
        continue;
      }
      reduce_step<true>(src, S, a, x0, y0);
      store_next(S, a, x0, y0, k);
      expand_blend_step<true>(src, S, a, x0, y0, acc);
    } else {
      // ---- load level-l Gaussian / support (G region) and mask (M region)
      const LevelPlanes& in = a.in[k];
      for (int i = threadIdx.x; i < GH * GW; i += blockDim.x) {
        int X = x0 - 4 + i % GW, Y = y0 - 4 + i / GW;
        bool inb = X >= 0 && Y >= 0 && X < a.wl && Y < a.hl;
        int64_t o = (int64_t)Y * a.pitch_l + X;
        spl[i] = inb ? in.s[o] : 0;
        for (int c = 0; c < 3; ++c) gpl[c * GH * GW + i] = inb ? in.g[c * in.plane + o] : 0.0f;
      }
      for (int i = threadIdx.x; i < MH * MW; i += blockDim.x) {
        int X = x0 - 2 + i % MW, Y = y0 - 2 + i / MW;
        bool inb = X >= 0 && Y >= 0 && X < a.wl && Y < a.hl;
        S.m[i] = inb ? in.m[(int64_t)Y * a.pitch_l + X] : 0.0f;
      }
      __syncthreads();
      GSource<false> src;
      src.gp = gpl;
      src.sp = spl;
      reduce_step<false>(src, S, a, x0, y0);
      store_next(S, a, x0, y0, k);
      expand_blend_step<false>(src, S, a, x0, y0, acc);
    }
  }
#pragma unroll
  for (int i = 0; i < kPPT; ++i) {
    int p = threadIdx.x + i * kThreads;
    int X = x0 + p % kTileW, Y = y0 + p / kTileW;
    if (X < a.wl && Y < a.hl) {
      int64_t o = (int64_t)Y * a.pitch_l + X;
#pragma unroll
      for (int c = 0; c < 3; ++c) a.acc_l[c * a.acc_plane_l + o] = acc[i][c];
    }
  }
}

cudaError_t launch_level0(const LevelArgs& a, cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(level_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  dim3 grid((a.wl + kTileW - 1) / kTileW, (a.hl + kTileH - 1) / kTileH);
  level_kernel<true><<<grid, kThreads, level0_smem_bytes(a.border), s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_level(const LevelArgs& a, cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(level_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  dim3 grid((a.wl + kTileW - 1) / kTileW, (a.hl + kTileH - 1) / kTileH);
  level_kernel<false><<<grid, kThreads, level_smem_bytes(), s>>>(a);
  return cudaGetLastError();
}

// ================================================================ collapse
// parent += EXPAND(child) in place (src/fuse/pyramid.zig:223-248); at level
// 0 also quantise trunc(clamp(v + 0.5, 0, 255)) into interleaved RGB.
__global__ void __launch_bounds__(kThreads) collapse_kernel(const __grid_constant__ CollapseArgs a) {
  __shared__ float cg[3][NH * NW];
  __shared__ float hrow[NH * kTileW * 3];
  const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * kTileH;
  const int x1 = x0 >> 1, y1 = y0 >> 1;
  const bool exact = a.exact_expand != 0;
  for (int i = threadIdx.x; i < NH * NW; i += blockDim.x) {
    int X = x1 - 1 + i % NW, Y = y1 - 1 + i / NW;
    bool in = X >= 0 && Y >= 0 && X < a.wc && Y < a.hc;
    int64_t o = (int64_t)Y * a.pitch_c + X;
    for (int c = 0; c < 3; ++c) cg[c][i] = in ? a.acc_c[c * a.plane_c + o] : 0.0f;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NH * kTileW; i += blockDim.x) {
    int ii = i / kTileW, xx = i % kTileW;
    int yi = y1 - 1 + ii;
    if (yi < 0 || yi >= a.hc) continue;
    for (int c = 0; c < 3; ++c) hrow[i * 3 + c] = expand_h(cg[c] + ii * NW, x0 + xx, x1, a.wc, exact);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kTileH * kTileW; i += blockDim.x) {
    int yy = i / kTileW, xx = i % kTileW;
    int x = x0 + xx, y = y0 + yy;
    if (x >= a.wp || y >= a.hp) continue;
    int64_t o = (int64_t)y * a.pitch_p + x;
    for (int c = 0; c < 3; ++c) {
      float v = expand_v(hrow, kTileW * 3, xx * 3 + c, x, y, y1, a.wc, a.hc, exact);
      float* p = a.acc_p + c * a.plane_p + o;
      float nv = __fadd_rn(*p, v);
      if (a.out) {
        float q8 = fminf(fmaxf(__fadd_rn(nv, 0.5f), 0.0f), 255.0f);
        a.out[(int64_t)y * a.out_pitch + (int64_t)x * 3 + c] = (uint8_t)q8;
        if (a.base) a.base[(int64_t)y * a.base_pitch + (int64_t)x * 3 + c] = nv;
      } else {
        *p = nv;
      }
    }
  }
}

cudaError_t launch_collapse(const CollapseArgs& a, cudaStream_t s) {
  dim3 grid((a.wp + kTileW - 1) / kTileW, (a.hp + kTileH - 1) / kTileH);
  collapse_kernel<<<grid, kThreads, 0, s>>>(a);
  return cudaGetLastError();
}

// Quantise a single-level accumulator (1x1 images have no collapse step).
__global__ void quantize_kernel(const float* acc, int64_t plane, int64_t pitch, int w, int h, uint8_t* out,
                                int64_t out_pitch, float* base, int64_t base_pitch) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w * h) return;
  int x = i % w, y = i / w;
  for (int c = 0; c < 3; ++c) {
    float v = acc[c * plane + (int64_t)y * pitch + x];
    out[(int64_t)y * out_pitch + x * 3 + c] = (uint8_t)fminf(fmaxf(__fadd_rn(v, 0.5f), 0.0f), 255.0f);
    if (base) base[(int64_t)y * base_pitch + x * 3 + c] = v;
  }
}

cudaError_t launch_quantize(const float* acc, int64_t plane, int64_t pitch, int w, int h, uint8_t* out,
                            int64_t out_pitch, float* base, int64_t base_pitch, cudaStream_t s) {
  quantize_kernel<<<(w * h + 255) / 256, 256, 0, s>>>(acc, plane, pitch, w, h, out, out_pitch, base, base_pitch);
  return cudaGetLastError();
}

// ========================================================== mask support
// Support of the mask pyramid (frame independent): a level-(l+1) sample is
// supported when any in-range 5x5 tap below it is (src/fuse/pyramid.zig:1032-1040).
__global__ void mask_support_kernel(const __grid_constant__ MaskSupportArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.dw * a.dh) return;
  int x = i % a.dw, y = i / a.dw;
  uint8_t any = 0;
  for (int ky = 0; ky < 5 && !any; ++ky) {
    int sy = 2 * y - 2 + ky;
    if (sy < 0 || sy >= a.sh) continue;
    for (int kx = 0; kx < 5; ++kx) {
      int sx = 2 * x - 2 + kx;
      if (sx < 0 || sx >= a.sw) continue;
      if (a.src[(int64_t)sy * a.spitch + sx]) {
        any = 1;
        break;
      }
    }
  }
  a.dst[(int64_t)y * a.dpitch + x] = any;
}

cudaError_t launch_mask_support(const MaskSupportArgs& a, cudaStream_t s) {
  int n = a.dw * a.dh;
  mask_support_kernel<<<(n + 255) / 256, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// ============================================================ remap only
// Standalone remap (src/remap.zig:166-278): ROI-sized output with
// channels + 1 samples per pixel.
__global__ void __launch_bounds__(kThreads) remap_kernel(const __grid_constant__ RemapArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * kTileH;
  const int nbx = kTileW / 8, nby = kTileH / 4, nb = nbx * nby;
  const bool fast_ok = a.f.warp.kind == WARP_HOMOGRAPHY && !a.f.warp.guard;
  const int du = lane & 7, dv = lane >> 3;
  for (int g0 = warp; g0 < nb; g0 += nwarps * 32) {
    Anchor mine = {};
    bool mine_ok = false;
    {
      const int bj = g0 + lane * nwarps;
      if (fast_ok && bj < nb) mine = make_anchor(a.f.warp, x0 + (bj % nbx) * 8, y0 + (bj / nbx) * 4, &mine_ok);
    }
    const int cnt = min(32, (nb - g0 + nwarps - 1) / nwarps);
    for (int j = 0; j < cnt; ++j) {
      const int blk = g0 + j * nwarps;
      const int AX = x0 + (blk % nbx) * 8, AY = y0 + (blk / nbx) * 4;
      const bool aok = __shfl_sync(0xffffffffu, mine_ok ? 1 : 0, j) != 0;
      const Anchor an = shfl_anchor(mine, j);
      const int X = AX + du, Y = AY + dv;
      if (X >= a.W || Y >= a.H) continue;
      uint32_t v = aok ? sample_fast(a.f.warp, a.f.src, an, du, dv, X, Y) : sample_exact(a.f.warp, a.f.src, X, Y);
      uint8_t* d = a.dst + (int64_t)Y * a.dst_pitch + (int64_t)X * a.dst_ch;
      if (a.dst_ch == 4) {
        d[0] = v & 255u;
        d[1] = (v >> 8) & 255u;
        d[2] = (v >> 16) & 255u;
        d[3] = v >> 24;
      } else {
        d[0] = v & 255u;
        d[1] = v >> 24;
      }
    }
  }
}

cudaError_t launch_remap(const RemapArgs& a, cudaStream_t s) {
  dim3 grid((a.W + kTileW - 1) / kTileW, (a.H + kTileH - 1) / kTileH);
  remap_kernel<<<grid, kThreads, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace fs
