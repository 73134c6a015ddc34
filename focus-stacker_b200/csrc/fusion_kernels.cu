// sm_100a kernels of the remap + pyramid-contrast fusion path.
//
// remap_weights_kernel<B>  remap (or aligned input) -> gray -> local contrast
//                          (window 2B+1) -> alpha weight; pass 1 adds it to
//                          the weight sum (frame order) and union support and
//                          can keep the remapped frame + weight for pass 2
// Pass 2 of the batch modes (CACHE / RESIDENT / REFETCH):
// level0_kernel            normalise the weights -> level-0 mask; REDUCE of
//                          frame and mask to level 1; EXPAND back; Laplacian
//                          x mask into the level-0 accumulator
// level_kernel<T>          the same step for level l >= 1 from HBM planes
//                          stored as T (f32 / f16 / bf16)
// The split pyramid (LAPS mode):
// lap0_kernel<B>           pass 1, level 0 fused: remap -> weight -> level-1
//                          Gaussian REDUCE -> EXPAND -> sum over frames of
//                          Laplacian x weight (divided by the weight sum in
//                          pass 2, finalize0_kernel)
// img_stream_kernel<T>     pass 1, each frame's Gaussian REDUCE and Laplacian
//                          on the clamped-EXPAND levels >= 1, streaming down
//                          column strips without shared memory
// img_kernel<T>            the same on the small (no-wrap) levels, per tile
// mask_reduce_kernel       each frame's mask pyramid, one level per launch
//                          (level 0 normalises the weights on the fly)
// blend_kernel<T>          the blend of one level l >= 1 over every frame
// img_tail_kernel<T>       pass 1, the image pyramid of the small levels
//                          (sides <= 64) of a batch, one frame per CTA
// mask_tail_kernel<T>      pass 2, each frame's masks of the small levels
// blend_tail_kernel<T>     pass 2, the small levels' blends, then (last CTA)
//                          their collapse down to the first small level
// Both:
// collapse_kernel          parent += EXPAND(child); quantise at level 0
//
// All of it is stencil work on CUDA cores (no tensor cores).  The tile
// kernels stage 64x32 output tiles in shared memory with their halos, the
// frames of a batch (K <= 8) inside one CTA so that per-pixel state (weight
// sums, accumulators) is read and written once per batch; the streaming
// kernels keep their windows in registers.  Every FP32 sum keeps the
// reference's frame order.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstddef>
#include <type_traits>

#include "fusion_kernels.cuh"

namespace fs {

// cudaFuncSetAttribute acts on the current device: a kernel's raised
// dynamic shared-memory limit is remembered per device (ordinals below 64;
// larger ones set it on every launch), so that one process can drive
// several GPUs, from several threads.
struct DeviceOnce {
  std::atomic<uint64_t> done{0};
  template <class F>
  cudaError_t run(F&& set) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = dev >= 0 && dev < 64 ? (1ull << dev) : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = set();
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_release);
    return e;
  }
};

// Raise a kernel's dynamic shared-memory limit once per device.
template <typename K>
static cudaError_t configure(K kernel, size_t bytes, DeviceOnce* done) {
  return done->run([&] { return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes); });
}

namespace {

constexpr int TW = kTileW, TH = kTileH, NT = kThreads;
constexpr int PPT = TW * TH / NT;  // output pixels per thread
static_assert((NT / TW) * PPT == TH, "accumulator strips cover the tile");
// Tile pixel (row-major index) of a thread's i-th accumulator: each thread
// owns a column strip of PPT consecutive rows (column tid % TW), so that the
// vertical EXPAND of neighbouring rows shares its source rows in registers.
__device__ __forceinline__ int acc_pixel(int i) {
  return ((int)(threadIdx.x / TW) * PPT + i) * TW + (int)(threadIdx.x % TW);
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ float kw(int i) { return (i == 0 || i == 4) ? 1.0f : ((i == 1 || i == 3) ? 4.0f : 6.0f); }
__device__ __forceinline__ uint32_t px_alpha(uint32_t v) { return v >> 24; }
// channel c of a packed pixel as an exact float: the byte is placed under
// the exponent of 2^23 and 2^23 is subtracted
__device__ __forceinline__ float chf(uint32_t v, int c) {
  return __uint_as_float(__byte_perm(v, 0x4B000000u, 0x7440u + (unsigned)c)) - 8388608.0f;
}
// contrast word (16 bits): gray sum k = R + G + B (<= 765) in bits 0..14
// and the support flag at bit 15, zero for unsupported pixels, so that the
// sum of a window row of these words adds counts and gray sums in one
// integer add (a row of at most 15 words keeps its gray sum below 2^15)
__device__ __forceinline__ uint32_t contrast_word(uint32_t v) {
  if (px_alpha(v) == 0) return 0u;
  uint32_t k = (v & 255u) + ((v >> 8) & 255u) + ((v >> 16) & 255u);
  return k | kSupportFlag;
}

// A window-row sum of contrast words (count << 15 | gray sum) in the layout
// of the window sums, count << 20 | gray sum (a 15 x 15 window stays below
// 2^20 for the gray sum and 2^12 for the count)
__device__ __forceinline__ uint32_t row_sum_word(uint32_t p) { return p + (p >> 15) * ((1u << 20) - kSupportFlag); }

// Horizontal window sums of one region row for 8 consecutive output columns:
// h1 = count << 20 | gray sum and h2 = sum of gray^2 over the window
// columns [c, c + 2B], sliding from the first column
template <int B>
__device__ __forceinline__ void window_row8(const uint16_t* row, uint32_t* h1, uint32_t* h2) {
  uint32_t p = 0, q = 0;
#pragma unroll
  for (int t = 0; t <= 2 * B; ++t) {
    const uint32_t v = row[t];
    const uint32_t g = v & 0x7FFFu;
    p += v;
    q += g * g;
  }
  h1[0] = row_sum_word(p);
  h2[0] = q;
#pragma unroll
  for (int c = 1; c < 8; ++c) {
    const uint32_t vin = row[c + 2 * B], vout = row[c - 1];
    const uint32_t gin = vin & 0x7FFFu, gout = vout & 0x7FFFu;
    p += vin - vout;
    q += gin * gin - gout * gout;
    h1[c] = row_sum_word(p);
    h2[c] = q;
  }
}

// Row stride (elements) of a region's 16-bit contrast words: an odd number of
// 32-bit words, so that threads on consecutive rows hit distinct banks.
constexpr int kv_stride(int rw) { return ((rw + 1) / 2) % 2 == 1 ? 2 * ((rw + 1) / 2) : 2 * ((rw + 1) / 2) + 2; }

// f32(alpha) / 255 as the reference computes it (src/fuse/masks.zig:18).
__device__ __forceinline__ float alpha_support(uint32_t al) {
  return al == 255u ? 1.0f : __fdiv_rn((float)al, 255.0f);
}

// Sample standard deviation of gray = k / 765 over the supported pixels of
// the window, from exact integer sums (src/fuse/contrast.zig:284-290):
// var = (n S2 - S1^2) / (n (n - 1) 765^2); inv_den[n] = 1 / (n (n-1) 765^2).
// Without branches: inv_den[0] = inv_den[1] = 0 and a nonpositive numerator
// clamped to 0 give the 0 of a window with fewer than two samples or no
// spread.
template <int B>
__device__ __forceinline__ float window_stddev(uint32_t packed, uint32_t s2, const float* inv_den) {
  const int n = (int)(packed >> 20);
  const int s1 = (int)(packed & 0xFFFFFu);
  float num;
  if (B <= 3) {
    num = (float)max(n * (int)s2 - s1 * s1, 0);  // < 2^31 for windows up to 7x7
  } else {
    num = (float)max((long long)n * s2 - (long long)s1 * s1, 0ll);
  }
  return sqrtf(num * inv_den[n]);
}

// ------------------------------------------------- region of a tile
constexpr int kExactQueue = 256;  // deferred exact samples per CTA and frame
constexpr int32_t kNoAnchor = INT32_MIN;

// Rows [y0 - R0, y0 - R0 + RH) x columns [x0 - R0, x0 - R0 + RW) of a frame's
// RGBA plane (written by remap_tile_kernel; 16-byte aligned rows) into
// shared memory: the packed words into `reg` (row stride RW) and their
// 16-bit contrast words into `kv` (row stride KS), zero outside the ROI.
// The rows are read in 16-byte chunks from column x0 - CB (R0 rounded up to
// a multiple of 4).
template <int RW, int RH, int KS, int R0>
__device__ __forceinline__ void load_region(const uint32_t* plane, int64_t pitch, int W, int H, int x0, int y0,
                                            uint32_t* reg, uint16_t* kv) {
  constexpr int CB = (R0 + 3) / 4 * 4;
  constexpr int SK = CB - R0;  // chunk columns before the region's first
  constexpr int CHUNKS = (RW + SK + 3) / 4;
  for (int it = threadIdx.x; it < RH * CHUNKS; it += NT) {
    const int r = it / CHUNKS, c = it - r * CHUNKS;
    const int Y = y0 - R0 + r, Xc = x0 - CB + 4 * c;
    uint4 q = make_uint4(0u, 0u, 0u, 0u);
    if ((unsigned)Y < (unsigned)H && Xc >= 0 && Xc < W) {
      q = __ldg(reinterpret_cast<const uint4*>(plane + (int64_t)Y * pitch + Xc));
      if (Xc + 3 >= W) {  // words past the last column are not samples
        if (Xc + 1 >= W) q.y = 0u;
        if (Xc + 2 >= W) q.z = 0u;
        q.w = 0u;
      }
    }
    const uint32_t wv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int rc = 4 * c + e - SK;
      if ((SK == 0 || rc >= 0) && rc < RW) {
        reg[r * RW + rc] = wv[e];
        kv[r * KS + rc] = (uint16_t)contrast_word(wv[e]);
      }
    }
  }
}

}  // namespace

// ======================================================== remap + weights
// Pass 1 in two kernels per batch of K frames:
//  remap_tile_kernel   one frame per grid z: each 64x32 tile's samples,
//                      written as packed RGBA words (the kept plane, or the
//                      batch slot when the mode keeps none); no halo, so
//                      every sample is taken once;
//  weights_kernel<B>   each tile with its window halo read back from those
//                      planes (L2), contrast words, sliding window sums, the
//                      alpha-weighted standard deviation; pass 1 adds it to
//                      the weight sum (frame order) and union support.

namespace {

constexpr int kTileBlocks = (TW / 8) * (TH / 4);  // 8x4 anchor blocks of a tile
constexpr int kRowsPerThread = TW * TH / NT;      // tile rows a thread samples (column fixed)
static_assert(NT % TW == 0 && (NT / TW) == 4 && kRowsPerThread * 4 == TH, "one anchor row per pass");

struct __align__(16) RemapTileSmem {
  TileAnchor anchor[kTileBlocks];
  uint32_t count;
  uint32_t overflow;
  uint32_t base;               // the CTA's first entry in the batch's exact-sample queue (kNoQueue: no room)
  uint32_t reserved;           // the first entry reserved when there was no room
  uint32_t item[kExactQueue];  // ry << 16 | rx
};
constexpr uint32_t kNoQueue = 0xFFFFFFFFu;
constexpr uint64_t kEmptyEntry = ~0ull;

}  // namespace

// Thread t samples column rx = t % 64 of the tile at rows t / 64 + 4 j, so
// its offsets (du, dv) inside the 8x4 blocks are fixed and block row j is
// pass j; samples the fast path cannot decide are queued and taken exactly
// after the pass (and, should the queue overflow, on a second pass).  CH:
// channels of remapped sources (3 or 1); aligned frames read theirs at run
// time.
template <int CH>
__global__ void __launch_bounds__(NT, 6) remap_tile_kernel(const __grid_constant__ RemapWeightArgs a) {
  __shared__ RemapTileSmem S;
  const int k = blockIdx.z;
  const FrameIn& f = a.f[k];
  uint32_t* const out = a.out[k].rgba;
  const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  const int rx = threadIdx.x % TW, ry0 = threadIdx.x / TW;
  const int X = x0 + rx;
  const int64_t pitch = a.pitch;
  // rows of this thread's column inside the ROI
  const int nrows = X < a.W ? min(kRowsPerThread, (a.H - y0 - ry0 + 3) / 4) : 0;
  uint32_t* const col = out + (int64_t)(y0 + ry0) * pitch + X;
  if (f.warp.kind == WARP_ALIGNED) {
    const int ch = f.src.ch;
    const uint8_t* p = f.src.px + (int64_t)(y0 + ry0) * f.src.pitch + (int64_t)X * ch;
    for (int j = 0; j < nrows; ++j, p += 4 * f.src.pitch) {
      const uint32_t al = ch == 4 ? (uint32_t)__ldg(p + 3) : 255u;
      col[4 * j * pitch] = pack_rgba(__ldg(p), __ldg(p + 1), __ldg(p + 2), al);
    }
    return;
  }
  if (threadIdx.x < kTileBlocks) {
    const bool fast_ok = f.warp.kind == WARP_HOMOGRAPHY && !f.warp.guard && f.src.w >= 4 && f.src.h >= 4;
    const int b = threadIdx.x;
    bool ok = false;
    Anchor an = {};
    if (fast_ok) an = make_anchor(f.warp, x0 + (b % (TW / 8)) * 8, y0 + (b / (TW / 8)) * 4, &ok);
    TileAnchor t = tile_anchor(an);
    if (!ok) t.kx = kNoTileAnchor;
    S.anchor[b] = t;
  }
  if (threadIdx.x == 0) {
    S.count = 0;
    S.overflow = 0;
  }
  __syncthreads();
  const int du = rx & 7, dv = ry0;
  const float fdu = (float)du, fdv = (float)dv;
  // the frame's pixel (1, 1): tap offsets are (x0 - 1, y0 - 1) from it
  const uint32_t spitch = (uint32_t)f.src.pitch;
  const uint8_t* const org = f.src.px + spitch + CH;
  const uint32_t xm = (uint32_t)(f.src.w - 4), ym = (uint32_t)(f.src.h - 4);
  const float lim = 0.5f - fmaxf(f.warp.tie_band, kTieBand);
  const TileAnchor* an_col = S.anchor + (rx >> 3);
  const int64_t step = 4 * pitch;
  auto undecided = [&](int j) {
    const uint32_t slot = atomicAdd(&S.count, 1u);
    if (slot < (uint32_t)kExactQueue) S.item[slot] = ((uint32_t)(ry0 + 4 * j) << 16) | (uint32_t)rx;
    else S.overflow = 1;
  };
  // two rows per step, both samples taken before either is stored, so that
  // their tap loads are in flight together
  for (int j = 0; j < nrows; j += 2) {
    const bool two = j + 1 < nrows;
    const TileAnchor an0 = an_col[j * (TW / 8)];
    const TileAnchor an1 = an_col[(two ? j + 1 : j) * (TW / 8)];
    uint32_t v0, v1;
    const bool ok0 = sample_tile<CH>(org, spitch, xm, ym, lim, an0, fdu, fdv, du, dv, &v0);
    const bool ok1 = sample_tile<CH>(org, spitch, xm, ym, lim, an1, fdu, fdv, du, dv, &v1);
    if (ok0) col[j * step] = v0;
    else undecided(j);
    if (two) {
      if (ok1) col[(j + 1) * step] = v1;
      else undecided(j + 1);
    }
  }
  __syncthreads();
  const uint32_t n = min(S.count, (uint32_t)kExactQueue);
  if (a.exact_q && !S.overflow && n > 0) {  // block-uniform
    // hand the undecided samples to the batch's queue: the exact FP64 sampler
    // then runs on full warps in remap_exact_kernel instead of on a few lanes
    // of this CTA while its other warps have finished
    if (threadIdx.x == 0) {
      const uint32_t base = atomicAdd(a.exact_n, n);
      S.base = base + n <= a.exact_cap ? base : kNoQueue;
      S.reserved = base;
    }
    __syncthreads();
    if (S.base != kNoQueue) {
      for (uint32_t i = threadIdx.x; i < n; i += NT) {
        const uint32_t qx = S.item[i] & 0xFFFFu, qy = S.item[i] >> 16;
        a.exact_q[S.base + i] = ((uint64_t)k << 48) | ((uint64_t)(y0 + qy) << 24) | (uint64_t)(x0 + qx);
      }
      return;
    }
    // no room: the entries reserved below the capacity stay empty and the
    // CTA takes its samples itself
    for (uint32_t i = threadIdx.x; i < n && S.reserved + i < a.exact_cap; i += NT)
      a.exact_q[S.reserved + i] = kEmptyEntry;
  }
  for (uint32_t i = threadIdx.x; i < n; i += NT) {
    const int qx = (int)(S.item[i] & 0xFFFFu), qy = (int)(S.item[i] >> 16);
    out[(int64_t)(y0 + qy) * pitch + x0 + qx] = sample_exact(f.warp, f.src, x0 + qx, y0 + qy);
  }
  if (S.overflow) {  // block-uniform: more undecided samples than the queue holds
    for (int j = 0; j < nrows; ++j) {
      const TileAnchor an = an_col[j * (TW / 8)];
      uint32_t v;
      if (!sample_tile<CH>(org, spitch, xm, ym, lim, an, fdu, fdv, du, dv, &v))
        col[j * step] = sample_exact(f.warp, f.src, X, y0 + ry0 + 4 * j);
    }
  }
}

// The batch's queued samples, one per thread, by the reference's FP64
// sampler (the same call the tile kernel makes for the samples it keeps).
__global__ void __launch_bounds__(NT) remap_exact_kernel(const __grid_constant__ RemapWeightArgs a) {
  const uint32_t n = min(*a.exact_n, a.exact_cap);
  for (uint32_t i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT) {
    const uint64_t e = a.exact_q[i];
    if (e == kEmptyEntry) continue;
    const int k = (int)(e >> 48), Y = (int)((e >> 24) & 0xFFFFFFu), X = (int)(e & 0xFFFFFFu);
    a.out[k].rgba[(int64_t)Y * a.pitch + X] = sample_exact(a.f[k].warp, a.f[k].src, X, Y);
  }
}

namespace {

// Weights kernel geometry: the region is the tile with the window halo B;
// its rows are read from the RGBA planes in 16-byte chunks of four words,
// and its contrast words kept from column x0 - CB on (CB = B rounded up to
// 4), so that every chunk lands whole (RX columns per row).
template <int B>
struct WLayout {
  static constexpr int RH = TH + 2 * B;
  static constexpr int CB = (B + 3) / 4 * 4;
  static constexpr int RX = TW + 2 * CB;
  static constexpr int CHUNKS = RX / 4;  // chunks per region row
  static constexpr int KS = kv_stride(RX), HS = TW + 1;
  static constexpr int NWIN = (2 * B + 1) * (2 * B + 1);
};

template <int B>
struct __align__(16) WeightsSmem {
  using Lay = WLayout<B>;
  uint16_t kv[Lay::RH * Lay::KS];   // contrast words of the region
  uint8_t alpha[TW * TH];           // alpha of the tile's samples
  uint32_t h1[Lay::RH * Lay::HS];   // horizontal window sums: count << 20 | gray sum
  uint32_t h2[Lay::RH * Lay::HS];   // sum of gray^2
  float asup[256];                  // alpha support f32(a) / 255
  float inv_den[Lay::NWIN + 1];
};

// Contrast words of two packed samples as one 32-bit pair (first in the low
// half), in 16-bit lanes: gray sums of the bytes, support flag where alpha
// is nonzero, zero where it is zero.
__device__ __forceinline__ uint32_t contrast_pair(uint32_t v0, uint32_t v1) {
  const uint32_t r = __byte_perm(v0, v1, 0x7470u) & 0x00FF00FFu;  // R0, R1 in lanes
  const uint32_t g = __byte_perm(v0, v1, 0x7571u) & 0x00FF00FFu;
  const uint32_t b = __byte_perm(v0, v1, 0x7672u) & 0x00FF00FFu;
  const uint32_t al = __byte_perm(v0, v1, 0x7773u) & 0x00FF00FFu;
  const uint32_t flag = (al + 0x7FFF7FFFu) & 0x80008000u;  // bit 15 of a lane set iff its alpha >= 1
  const uint32_t keep = (flag >> 15) * 0xFFFFu;            // the lane's mask
  return ((r + g + b) & keep) | flag;
}

}  // namespace

template <int B>
__global__ void __launch_bounds__(NT, 6) weights_kernel(const __grid_constant__ RemapWeightArgs a) {
  using Lay = WLayout<B>;
  constexpr int RH = Lay::RH, KS = Lay::KS, HS = Lay::HS, CB = Lay::CB, CHUNKS = Lay::CHUNKS;
  static_assert(kSupportFlag == 0x8000u, "contrast_pair writes the flag at bit 15");
  extern __shared__ __align__(16) uint8_t smem_w[];
  WeightsSmem<B>& S = *reinterpret_cast<WeightsSmem<B>*>(smem_w);
  const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  for (int n = threadIdx.x; n <= Lay::NWIN; n += NT)
    S.inv_den[n] = n > 1 ? 1.0f / ((float)(n * (n - 1)) * 585225.0f) : 0.0f;
  for (int n = threadIdx.x; n < 256; n += NT) S.asup[n] = alpha_support((uint32_t)n);
  // own pixels: column vc, rows vr0 .. vr0 + 7; rows_in / win_rows: in the
  // ROI / with the whole window inside it (the reference's window rule)
  const int vc = threadIdx.x % TW, vr0 = (threadIdx.x / TW) * PPT;
  const int X = x0 + vc;
  const int64_t obase = (int64_t)(y0 + vr0) * a.pitch + X;
  float nacc[PPT];
  uint32_t umask = 0, rows_in = 0, win_rows = 0;
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    const int Y = y0 + vr0 + i;
    nacc[i] = 0.0f;
    if (X < a.W && Y < a.H) {
      rows_in |= 1u << i;
      if (a.window_ok && X >= B && Y >= B && X < a.W - B && Y < a.H - B) win_rows |= 1u << i;
      if (a.accumulate && !a.first) {
        nacc[i] = a.norm[obase + (int64_t)i * a.pitch];
        if (a.uni[obase + (int64_t)i * a.pitch]) umask |= 1u << i;
      }
    }
  }
  const bool right_edge = x0 + TW + CB > a.W;  // chunks reaching past the ROI's last column
  for (int k = 0; k < a.K; ++k) {
    const uint32_t* plane = a.out[k].rgba;
    // region rows -> contrast words (0 outside the ROI) and the tile's alpha
    for (int it = threadIdx.x; it < RH * CHUNKS; it += NT) {
      const int r = it / CHUNKS, c = it - r * CHUNKS;
      const int Y = y0 - B + r, Xc = x0 - CB + 4 * c;  // first column of the chunk
      uint4 q = make_uint4(0u, 0u, 0u, 0u);
      if ((unsigned)Y < (unsigned)a.H && Xc >= 0 && Xc < a.W) {
        q = __ldg(reinterpret_cast<const uint4*>(plane + (int64_t)Y * a.pitch + Xc));
        if (right_edge) {  // words past the last column are not samples
          if (Xc + 1 >= a.W) q.y = 0u;
          if (Xc + 2 >= a.W) q.z = 0u;
          if (Xc + 3 >= a.W) q.w = 0u;
        }
      }
      uint32_t* kw = reinterpret_cast<uint32_t*>(S.kv + r * KS + 4 * c);
      kw[0] = contrast_pair(q.x, q.y);
      kw[1] = contrast_pair(q.z, q.w);
      const int ar = r - B, ac = 4 * c - CB;
      if ((unsigned)ar < (unsigned)TH && (unsigned)ac < (unsigned)TW)
        *reinterpret_cast<uint32_t*>(S.alpha + ar * TW + ac) =
            __byte_perm(__byte_perm(q.x, q.y, 0x0073u), __byte_perm(q.z, q.w, 0x0073u), 0x5410u);
    }
    __syncthreads();
    // rows 0..31 first, a warp per column block, then the RH - 32 halo rows:
    // the lanes of a warp never wrap to a second column block, whose rows
    // would fall on the same shared-memory banks
    static_assert(NT == 32 * (TW / 8), "one pass covers rows 0..31 of every column block");
    for (int it = threadIdx.x; it < RH * (TW / 8); it += NT) {
      int r, c0;
      if (it < NT) {
        r = it % 32;
        c0 = (it / 32) * 8;
      } else {
        r = 32 + (it - NT) % (RH - 32);
        c0 = ((it - NT) / (RH - 32)) * 8;
      }
      window_row8<B>(S.kv + r * KS + c0 + CB - B, S.h1 + r * HS + c0, S.h2 + r * HS + c0);
    }
    __syncthreads();
    {
      uint32_t p = 0, q = 0;
#pragma unroll
      for (int t = 0; t <= 2 * B; ++t) {
        p += S.h1[(vr0 + t) * HS + vc];
        q += S.h2[(vr0 + t) * HS + vc];
      }
      float* const wout = a.out[k].w;
#pragma unroll
      for (int i = 0; i < PPT; ++i) {
        if (i > 0) {
          p += S.h1[(vr0 + i + 2 * B) * HS + vc] - S.h1[(vr0 + i - 1) * HS + vc];
          q += S.h2[(vr0 + i + 2 * B) * HS + vc] - S.h2[(vr0 + i - 1) * HS + vc];
        }
        const uint32_t al = S.alpha[(vr0 + i) * TW + vc];
        // alpha 0 has support 0: the weight is 0 without a test
        const float w = ((win_rows >> i) & 1u) ? __fmul_rn(window_stddev<B>(p, q, S.inv_den), S.asup[al]) : 0.0f;
        if (a.accumulate) {
          nacc[i] = __fadd_rn(nacc[i], w);
          umask |= (al > 0 ? 1u : 0u) << i;
        }
        if (wout && ((rows_in >> i) & 1u)) wout[obase + (int64_t)i * a.pitch] = w;
      }
    }
    __syncthreads();
  }
  if (a.accumulate) {
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      if ((rows_in >> i) & 1u) {
        a.norm[obase + (int64_t)i * a.pitch] = nacc[i];
        a.uni[obase + (int64_t)i * a.pitch] = (uint8_t)((umask >> i) & 1u);
      }
    }
  }
}

template <int B>
static cudaError_t launch_weights(const RemapWeightArgs& a, cudaStream_t s) {
  static DeviceOnce configured;
  const size_t sm = sizeof(WeightsSmem<B>);
  cudaError_t e = configure(weights_kernel<B>, sm, &configured);
  if (e != cudaSuccess) return e;
  dim3 grid((a.W + TW - 1) / TW, (a.H + TH - 1) / TH);
  weights_kernel<B><<<grid, NT, sm, s>>>(a);
  return cudaGetLastError();
}

// Every frame's plane must hold RGBA words (the weights read them back) on
// 16-byte aligned rows; remapped frames stay below 4 GiB (32-bit tap
// offsets).  The frames of a batch share their channel count: the remap
// kernel has it compiled in (RGB or gray; aligned frames read it).
cudaError_t launch_remap_tiles(const RemapWeightArgs& a, cudaStream_t s) {
  if (a.K < 1 || a.K > kMaxBatch || a.W < 1 || a.H < 1 || (a.pitch & 3)) return cudaErrorInvalidValue;
  for (int k = 0; k < a.K; ++k) {
    if (!a.out[k].rgba || ((uintptr_t)a.out[k].rgba & 15)) return cudaErrorInvalidValue;
    const SrcImage& src = a.f[k].src;
    if (a.f[k].warp.kind != WARP_ALIGNED && (src.ch != a.f[0].src.ch || (src.ch != 1 && src.ch != 3) ||
                                             (uint64_t)src.pitch * (uint64_t)src.h >= (1ull << 32)))
      return cudaErrorInvalidValue;
  }
  if (a.exact_q && (!a.exact_n || ((uintptr_t)a.exact_q & 7))) return cudaErrorInvalidValue;
  if (a.exact_q) {
    cudaError_t e = cudaMemsetAsync(a.exact_n, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
  }
  const dim3 grid((a.W + TW - 1) / TW, (a.H + TH - 1) / TH, a.K);
  if (a.f[0].src.ch == 1) remap_tile_kernel<1><<<grid, NT, 0, s>>>(a);
  else remap_tile_kernel<3><<<grid, NT, 0, s>>>(a);
  if (a.exact_q) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    remap_exact_kernel<<<(unsigned)(8 * sms), NT, 0, s>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_remap_weights(const RemapWeightArgs& a, int border, cudaStream_t s) {
  cudaError_t e = launch_remap_tiles(a, s);
  if (e != cudaSuccess) return e;
  switch (border) {
    case 1: return launch_weights<1>(a, s);
    case 2: return launch_weights<2>(a, s);
    case 3: return launch_weights<3>(a, s);
    case 4: return launch_weights<4>(a, s);
    case 5: return launch_weights<5>(a, s);
    case 6: return launch_weights<6>(a, s);
    case 7: return launch_weights<7>(a, s);
    default: return cudaErrorInvalidValue;
  }
}

// =========================================================== level kernels
// Shared-memory geometry of one level step (tile origin x0, y0 at level l;
// level-(l+1) tile origin x1 = x0 / 2, y1 = y0 / 2):
//   G region   level-l cols [x0 - 4, x0 + TW + 2], rows [y0 - 4, y0 + TH + 2]
//              (feeds level-(l+1) Gaussians on the tile plus a 1-pixel halo,
//              which the expand back to the tile needs)
//   M region   level-l cols [x0 - 2, x0 + TW], rows [y0 - 2, y0 + TH]
//              (feeds the level-(l+1) mask on the tile)
//   N tile     level-(l+1) cols [x1 - 1, x1 + TW/2], rows [y1 - 1, y1 + TH/2]
// Samples outside the level are staged with support 0 (and value 0), so the
// support-weighted REDUCE needs no bounds tests: a zero-support tap adds
// nothing, exactly like the reference's skipped taps.
namespace {

constexpr int GW = TW + 7, GH = TH + 7;          // G region
constexpr int MW = TW + 3, MH = TH + 3;          // M region
constexpr int NW = TW / 2 + 2, NH = TH / 2 + 2;  // level l+1 tile + halo
constexpr int TW1 = TW / 2, TH1 = TH / 2;
// Row strides of the REDUCE temporaries, padded so that lanes on
// consecutive rows hit distinct shared-memory banks.
constexpr int THS = NW + 1;   // horizontal image sums (float4)
constexpr int TMS = TW1 + 1;  // horizontal mask sums (float2)
constexpr int kTmpFloats = (GH * THS * 4 > NH * TW * 3) ? GH * THS * 4 : NH * TW * 3;

struct __align__(16) LevelSmem {
  static constexpr int kTmOffset = kTmpFloats - MH * TMS * 2;  // mask REDUCE rows at the end of tmp
  float4 gs[GH * GW];       // level-l Gaussian (r, g, b) and support (0 / 1)
  float tmp[kTmpFloats];    // reduce / expand temporaries
  float ng[3][NH * NW];     // level-(l+1) Gaussian (zero outside the level)
  float nm[TH1 * TW1];      // level-(l+1) mask on the tile
  float m[MH * MW];         // level-l mask (M region)
  uint8_t sm[MH * MW];      // level-l mask support (M region)
  uint8_t ns[NH * NW];      // level-(l+1) support
};
static_assert(offsetof(LevelSmem, tmp) % 16 == 0, "tmp is accessed as float4");

template <typename T> __device__ __forceinline__ float ldv(const T* p, int64_t i);
template <> __device__ __forceinline__ float ldv<float>(const float* p, int64_t i) { return p[i]; }
template <> __device__ __forceinline__ float ldv<__half>(const __half* p, int64_t i) { return __half2float(p[i]); }
template <> __device__ __forceinline__ float ldv<__nv_bfloat16>(const __nv_bfloat16* p, int64_t i) {
  return __bfloat162float(p[i]);
}
template <typename T> __device__ __forceinline__ void stv(T* p, int64_t i, float v);
template <> __device__ __forceinline__ void stv<float>(float* p, int64_t i, float v) { p[i] = v; }
template <> __device__ __forceinline__ void stv<__half>(__half* p, int64_t i, float v) { p[i] = __float2half_rn(v); }
template <> __device__ __forceinline__ void stv<__nv_bfloat16>(__nv_bfloat16* p, int64_t i, float v) {
  p[i] = __float2bfloat16_rn(v);
}

// EXPAND taps.  clamped (parent larger than 512), src/fuse/pyramid.zig:
// 1101-1149, 1748-1775: even 2j uses s[j-1], s[j], s[j+1] -> (a + 6b + c) / 8,
// odd 2j+1 uses s[j], s[j+1] -> (a + b) / 2, coordinates clamped; vertically
// the odd row 2i+1 reads row i twice (src/fuse/pyramid.zig:1122-1145).
// no-wrap (parent at most 512), src/fuse/pyramid.zig:1167-1354: the same taps
// with zero outside, (a + 6b) + c and 4 (a + b) horizontally, (a + 6b) + c and
// a + b vertically, then one division by the position-dependent normaliser.
// Every operation is in the reference's order, so both modes are bit-exact.
struct Taps {
  int i0, i1, i2;   // local indices (i2 unused for odd)
  bool odd;
};
__device__ __forceinline__ Taps expand_taps(int x, int c1, int wc, bool exact) {
  const int j = x >> 1, o = c1 - 1;
  Taps t;
  t.odd = (x & 1) != 0;
  if (exact) {
    t.i0 = t.odd ? j - o : j - 1 - o;
    t.i1 = t.odd ? j + 1 - o : j - o;
    t.i2 = j + 1 - o;
  } else {
    t.i0 = (t.odd ? clampi(j, 0, wc - 1) : clampi(j - 1, 0, wc - 1)) - o;
    t.i1 = (t.odd ? clampi(j + 1, 0, wc - 1) : clampi(j, 0, wc - 1)) - o;
    t.i2 = clampi(j + 1, 0, wc - 1) - o;
  }
  return t;
}
__device__ __forceinline__ float expand_h1(const float* g, const Taps& t, bool exact) {
  if (exact) {
    if (t.odd) return __fmul_rn(4.0f, __fadd_rn(g[t.i0], g[t.i1]));
    return __fadd_rn(__fadd_rn(g[t.i0], __fmul_rn(6.0f, g[t.i1])), g[t.i2]);
  }
  if (t.odd) return __fmul_rn(__fadd_rn(g[t.i0], g[t.i1]), 0.5f);
  return __fmul_rn(__fadd_rn(__fadd_rn(g[t.i0], __fmul_rn(6.0f, g[t.i1])), g[t.i2]), 0.125f);
}
// vertical rows of output row y (local row indices of the horizontal stage),
// -1 for a zero row of the no-wrap mode
struct Rows {
  int r0, r1, r2;
  bool odd;
};
__device__ __forceinline__ Rows expand_rows(int y, int c1, int hc, bool exact) {
  const int q = y >> 1, o = c1 - 1;
  Rows r;
  r.odd = (y & 1) != 0;
  if (exact) {
    auto z = [&](int v) { return (v < 0 || v >= hc) ? -1 : v - o; };
    r.r0 = r.odd ? z(q) : z(q - 1);
    r.r1 = r.odd ? z(q + 1) : z(q);
    r.r2 = z(q + 1);
  } else {
    r.r0 = r.odd ? clampi(q, 0, hc - 1) - o : clampi(q - 1, 0, hc - 1) - o;
    r.r1 = r.odd ? r.r0 : clampi(q, 0, hc - 1) - o;
    r.r2 = clampi(q + 1, 0, hc - 1) - o;
  }
  return r;
}
__device__ __forceinline__ float expand_v1(const float* h, int stride, const Rows& r, bool exact, float div) {
  auto at = [&](int row) -> float { return row < 0 ? 0.0f : h[row * stride]; };
  if (exact) {
    float v = r.odd ? __fadd_rn(at(r.r0), at(r.r1))
                    : __fadd_rn(__fadd_rn(at(r.r0), __fmul_rn(6.0f, at(r.r1))), at(r.r2));
    return __fdiv_rn(v, div);
  }
  if (r.odd) {
    const float a = h[r.r0 * stride];
    return __fmul_rn(__fadd_rn(a, a), 0.5f);
  }
  return __fmul_rn(__fadd_rn(__fadd_rn(h[r.r0 * stride], __fmul_rn(6.0f, h[r.r1 * stride])), h[r.r2 * stride]),
                   0.125f);
}

// REDUCE with support to the level-(l+1) tile (+ halo for the Gaussian),
// src/fuse/pyramid.zig:997-1099: 5x5 taps [1 4 6 4 1]^2 over in-range
// samples with support > 0, value = sum(w v) / sum(w), support = sum(w) > 0.
// Evaluated separably (rows first); the weights are exact small integers.
template <class SM>
__device__ void reduce_image_step(SM& S, const LevelArgs& a, int x0, int y0) {
  const int x1 = x0 >> 1, y1 = y0 >> 1;
  float4* th = reinterpret_cast<float4*>(S.tmp);  // [GH][THS]
  // horizontal, two neighbouring outputs per thread (they share 3 of their
  // 5 taps); each output sums its taps in the same order as alone
  static_assert(NW % 2 == 0 && NH % 2 == 0 && TW1 % 2 == 0 && TH1 % 2 == 0, "output pairs");
  for (int i = threadIdx.x; i < GH * (NW / 2); i += NT) {
    const int ry = i % GH, jj = 2 * (i / GH);  // lanes on consecutive rows
    const float4* row = S.gs + ry * GW + 2 * jj;  // G region column of tap 0: 2j - 2 - (x0 - 4)
    float4 t[7];
#pragma unroll
    for (int u = 0; u < 7; ++u) t[u] = row[u];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float v0 = 0.f, v1 = 0.f, v2 = 0.f, ws = 0.f;
#pragma unroll
      for (int kx = 0; kx < 5; ++kx) {
        const float4 tk = t[2 * h + kx];
        const float w = kw(kx) * tk.w;
        v0 = fmaf(w, tk.x, v0);
        v1 = fmaf(w, tk.y, v1);
        v2 = fmaf(w, tk.z, v2);
        ws += w;
      }
      th[ry * THS + jj + h] = make_float4(v0, v1, v2, ws);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < (NH / 2) * NW; i += NT) {
    const int ii = 2 * (i / NW), jj = i % NW;
    const float4* col = th + (2 * ii) * THS + jj;  // G region row of tap 0: 2 yi - 2 - (y0 - 4)
    float4 t[7];
#pragma unroll
    for (int u = 0; u < 7; ++u) t[u] = col[u * THS];
    const int xj = x1 - 1 + jj;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int yi = y1 - 1 + ii + h;
      float v0 = 0.f, v1 = 0.f, v2 = 0.f, ws = 0.f;
#pragma unroll
      for (int ky = 0; ky < 5; ++ky) {
        const float4 tk = t[2 * h + ky];
        const float w = kw(ky);
        v0 = fmaf(w, tk.x, v0);
        v1 = fmaf(w, tk.y, v1);
        v2 = fmaf(w, tk.z, v2);
        ws = fmaf(w, tk.w, ws);
      }
      const bool sup = xj >= 0 && yi >= 0 && xj < a.wn && yi < a.hn && ws > 0.f;
      const float r = sup ? __fdividef(1.0f, ws) : 0.0f;
      const int o = (ii + h) * NW + jj;
      S.ng[0][o] = v0 * r;
      S.ng[1][o] = v1 * r;
      S.ng[2][o] = v2 * r;
      S.ns[o] = sup ? 1 : 0;
    }
  }
  __syncthreads();
}

// Mask half of the REDUCE (level-l mask with the level-l mask support).
template <class SM>
__device__ void reduce_mask_step(SM& S) {
  float2* tm = reinterpret_cast<float2*>(S.tmp + SM::kTmOffset);  // [MH][TMS]
  for (int i = threadIdx.x; i < MH * (TW1 / 2); i += NT) {
    const int ry = i % MH, jj = 2 * (i / MH);  // lanes on consecutive rows
    const int base = ry * MW + 2 * jj;  // M region column of tap 0: 2j - 2 - (x0 - 2)
    float mv[7], sw[7];
#pragma unroll
    for (int u = 0; u < 7; ++u) {
      mv[u] = S.m[base + u];
      sw[u] = S.sm[base + u] ? 1.0f : 0.0f;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float v = 0.f, ws = 0.f;
#pragma unroll
      for (int kx = 0; kx < 5; ++kx) {
        const float w = sw[2 * h + kx] != 0.0f ? kw(kx) : 0.0f;
        v = fmaf(w, mv[2 * h + kx], v);
        ws += w;
      }
      tm[ry * TMS + jj + h] = make_float2(v, ws);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < (TH1 / 2) * TW1; i += NT) {
    const int ii = 2 * (i / TW1), jj = i % TW1;
    float2 t[7];
#pragma unroll
    for (int u = 0; u < 7; ++u) t[u] = tm[(2 * ii + u) * TMS + jj];  // M region row of tap 0: 2 yi - 2 - (y0 - 2)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float v = 0.f, ws = 0.f;
#pragma unroll
      for (int ky = 0; ky < 5; ++ky) {
        const float w = kw(ky);
        v = fmaf(w, t[2 * h + ky].x, v);
        ws = fmaf(w, t[2 * h + ky].y, ws);
      }
      S.nm[(ii + h) * TW1 + jj] = ws > 0.f ? v * __fdividef(1.0f, ws) : 0.f;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void reduce_step(LevelSmem& S, const LevelArgs& a, int x0, int y0) {
  reduce_image_step(S, a, x0, y0);
  reduce_mask_step(S);
}

// Store the level-(l+1) tile (Gaussian, support, mask) of one frame, or add
// it into the top accumulator when l + 1 is the last level
// (src/fuse/pyramid.zig:1533-1554, 1605-1649).
template <typename T>
__device__ void store_next(const LevelSmem& S, const LevelArgs& a, int x0, int y0, int k) {
  const int x1 = x0 >> 1, y1 = y0 >> 1;
  const bool top = a.level + 1 == a.levels - 1;
  for (int i = threadIdx.x; i < TH1 * TW1; i += NT) {
    const int ii = i / TW1, jj = i % TW1;
    const int xj = x1 + jj, yi = y1 + ii;
    if (xj >= a.wn || yi >= a.hn) continue;
    const int ni = (ii + 1) * NW + (jj + 1);
    const int64_t o = (int64_t)yi * a.pitch_n + xj;
    if (top && a.frame_parallel) {
      const float m = S.nm[i];
#pragma unroll
      for (int c = 0; c < 3; ++c) a.contrib_top[(int64_t)(k * 3 + c) * a.acc_plane_n + o] = __fmul_rn(S.ng[c][ni], m);
    } else if (top) {
      const float m = S.nm[i];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float* acc = a.acc_n + c * a.acc_plane_n + o;
        *acc = __fadd_rn(*acc, __fmul_rn(S.ng[c][ni], m));
      }
    } else {
      const LevelPlanes& out = a.out[k];
      T* g = (T*)out.g;
#pragma unroll
      for (int c = 0; c < 3; ++c) stv<T>(g, c * out.plane + o, S.ng[c][ni]);
      out.s[o] = S.ns[ni];
      stv<T>((T*)out.m, o, S.nm[i]);
    }
  }
}

// EXPAND of the level-(l+1) Gaussian back to the level-l tile fused with the
// weighted Laplacian blend into the accumulator registers:
// acc += (G_l - EXPAND(G_{l+1})) * M_l  (src/fuse/pyramid.zig:1480-1504).
// LAP: store the Laplacian G_l - EXPAND(G_{l+1}) of the tile into lap (3
// planes of acc_plane_l floats, level pitch) instead of blending it.
template <bool LAP = false, class SM = LevelSmem, typename TL = float>
__device__ void expand_blend_step(SM& S, const LevelArgs& a, int x0, int y0, float (&acc)[PPT][3],
                                  TL* lap_out = nullptr) {
  const int x1 = x0 >> 1, y1 = y0 >> 1;
  float* hrow = S.tmp;  // [NH][3][TW]
  const bool exact = a.exact_expand != 0;
  // horizontal EXPAND, an even/odd output pair per thread: both read the
  // level-(l+1) columns j - 1, j, j + 1 (clamped, or zero outside the level
  // in the no-wrap mode), j = x / 2, with the operations of expand_h1
  for (int i = threadIdx.x; i < NH * (TW / 2); i += NT) {
    const int ii = i / (TW / 2), pp = i % (TW / 2);
    const int yi = y1 - 1 + ii;
    if (yi < 0 || yi >= a.hn) continue;
    const int j = x1 + pp, o = x1 - 1;
    int ia, ib, ic;
    if (exact) {
      ia = pp;
      ib = pp + 1;
      ic = pp + 2;
    } else {
      ia = clampi(j - 1, 0, a.wn - 1) - o;
      ib = clampi(j, 0, a.wn - 1) - o;
      ic = clampi(j + 1, 0, a.wn - 1) - o;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float* g = S.ng[c] + ii * NW;
      const float A = g[ia], B = g[ib], C = g[ic];
      float ev, od;
      if (exact) {
        ev = __fadd_rn(__fadd_rn(A, __fmul_rn(6.0f, B)), C);
        od = __fmul_rn(4.0f, __fadd_rn(B, C));
      } else {
        ev = __fmul_rn(__fadd_rn(__fadd_rn(A, __fmul_rn(6.0f, B)), C), 0.125f);
        od = __fmul_rn(__fadd_rn(B, C), 0.5f);
      }
      hrow[(ii * 3 + c) * TW + 2 * pp] = ev;
      hrow[(ii * 3 + c) * TW + 2 * pp + 1] = od;
    }
  }
  __syncthreads();
  // vertical EXPAND down this thread's strip: output rows yy0 .. yy0 + 7
  // (yy0 even) read level-(l+1) rows q0 - 1 .. q0 + 4, q0 = (y0 + yy0) / 2,
  // loaded once into registers (clamped rows for the clamped mode, zero
  // outside the level for the no-wrap mode; the same operands expand_rows
  // and expand_v1 select for each row)
  const int xx = threadIdx.x % TW, yy0 = (threadIdx.x / TW) * PPT;
  const int x = x0 + xx;
  const int q0 = (y0 + yy0) >> 1;
  constexpr int NR = PPT / 2 + 2;
  float hv[3][NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    int q = q0 - 1 + k;
    bool zero = false;
    if (exact) zero = q < 0 || q >= a.hn;
    else q = clampi(q, 0, a.hn - 1);
    const int lr = q - (y1 - 1);  // row of hrow
#pragma unroll
    for (int c = 0; c < 3; ++c) hv[c][k] = zero ? 0.0f : hrow[(lr * 3 + c) * TW + xx];
  }
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    const int yy = yy0 + i, y = y0 + yy;
    if (x >= a.wl || y >= a.hl) continue;
    const int j = i >> 1;
    const float div = exact ? exact_expand_divisor(x, y, a.wn, a.hn) : 1.0f;
    float m = 0.0f;
    if constexpr (!LAP) m = S.m[(yy + 2) * MW + (xx + 2)];
    const float4 g = S.gs[(yy + 4) * GW + (xx + 4)];
    const float gv[3] = {g.x, g.y, g.z};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float e;
      if ((i & 1) == 0) {  // even row: rows q - 1, q, q + 1
        const float v = __fadd_rn(__fadd_rn(hv[c][j], __fmul_rn(6.0f, hv[c][j + 1])), hv[c][j + 2]);
        e = exact ? __fdiv_rn(v, div) : __fmul_rn(v, 0.125f);
      } else if (exact) {  // odd row, no-wrap: rows q, q + 1
        e = __fdiv_rn(__fadd_rn(hv[c][j + 1], hv[c][j + 2]), div);
      } else {  // odd row, clamped: row q read twice
        e = __fmul_rn(__fadd_rn(hv[c][j + 1], hv[c][j + 1]), 0.5f);
      }
      const float lap = __fsub_rn(gv[c], e);
      if (LAP) stv<TL>(lap_out, c * a.acc_plane_l + (int64_t)y * a.pitch_l + x, lap);
      else acc[i][c] = __fadd_rn(acc[i][c], __fmul_rn(lap, m));
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void load_acc(const LevelArgs& a, int x0, int y0, float (&acc)[PPT][3]) {
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    const int p = acc_pixel(i);
    const int X = x0 + p % TW, Y = y0 + p / TW;
    const bool in = X < a.wl && Y < a.hl;
    const int64_t o = (int64_t)Y * a.pitch_l + X;
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[i][c] = in ? a.acc_l[c * a.acc_plane_l + o] : 0.0f;
  }
}
__device__ __forceinline__ void store_acc(const LevelArgs& a, int x0, int y0, const float (&acc)[PPT][3]) {
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    const int p = acc_pixel(i);
    const int X = x0 + p % TW, Y = y0 + p / TW;
    if (X < a.wl && Y < a.hl) {
      const int64_t o = (int64_t)Y * a.pitch_l + X;
#pragma unroll
      for (int c = 0; c < 3; ++c) a.acc_l[c * a.acc_plane_l + o] = acc[i][c];
    }
  }
}

template <class SM>
__device__ __forceinline__ void load_mask_support(SM& S, const LevelArgs& a, int x0, int y0) {
  for (int i = threadIdx.x; i < MH * MW; i += NT) {
    const int X = x0 - 2 + i % MW, Y = y0 - 2 + i / MW;
    const bool in = X >= 0 && Y >= 0 && X < a.wl && Y < a.hl;
    S.sm[i] = in ? a.sm_l[(int64_t)Y * a.pitch_l + X] : 0;
  }
}

}  // namespace

// Asynchronous global -> shared copies (cp.async, 16 B).  src_bytes < 16
// zero-fills the rest of the 16 bytes; with src_bytes == 0 nothing is read
// (the address given is still a valid one).
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Level-0 staging of one frame's pass-1 planes, copied while the previous
// frame is being reduced and blended.  Rows are 72 words wide starting at
// column x0 - 4 (16-byte aligned because x0 is a multiple of 64 and the level
// pitch a multiple of 32 words): G rows y0 - 4 .. y0 + TH + 2 of the RGBA
// words, M rows y0 - 2 .. y0 + TH of the weights.  Words outside the level are
// zero (alpha 0: no support).
constexpr int SW = 72, SCH = SW / 4;  // staged words per row, 16-byte chunks per row
struct __align__(16) Level0Smem {
  LevelSmem lv;
  uint32_t rgba[GH * SW];
  float w[MH * SW];
};
static_assert(offsetof(Level0Smem, rgba) % 16 == 0 && offsetof(Level0Smem, w) % 16 == 0, "cp.async targets");
static_assert(SW >= GW + 1 && TW % 4 == 0, "staging covers the G region");

__device__ __forceinline__ void stage_rows(void* dst, const void* plane, int64_t pitch, int x0, int ytop, int rows,
                                           int wl, int hl) {
  for (int i = threadIdx.x; i < rows * SCH; i += NT) {
    const int r = i / SCH, c = i % SCH;
    const int X = x0 - 4 + 4 * c, Y = ytop + r;
    int n = 0;
    const uint8_t* src = (const uint8_t*)plane;
    if (X >= 0 && Y >= 0 && Y < hl && X < wl) {
      n = min(4, wl - X) * 4;
      src += ((int64_t)Y * pitch + X) * 4;
    }
    cp_async16((uint8_t*)dst + (size_t)i * 16, src, n);
  }
}

__device__ __forceinline__ void stage_level0(Level0Smem& S, const LevelArgs& a, const FramePlanes& in, int x0,
                                             int y0) {
  stage_rows(S.rgba, in.rgba, a.pitch_l, x0, y0 - 4, GH, a.wl, a.hl);
  stage_rows(S.w, in.w, a.pitch_l, x0, y0 - 2, MH, a.wl, a.hl);
  cp_async_commit();
}

// Level 0 -> 1 for a batch of frames from their pass-1 planes (remapped RGBA
// and weight): mask = weight / sum (1/N where the sum is <= 1e-12,
// src/fuse/pyramid.zig:303-316), mask support = union.  Frame k + 1 is
// copied into the staging rows while frame k is reduced and blended.
template <typename T>
__global__ void __launch_bounds__(NT) level0_kernel(const __grid_constant__ LevelArgs a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  Level0Smem& S0 = *reinterpret_cast<Level0Smem*>(smem_raw);
  LevelSmem& S = S0.lv;
  const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  stage_level0(S0, a, a.in0[0], x0, y0);
  load_mask_support(S, a, x0, y0);
  float acc[PPT][3];
  load_acc(a, x0, y0, acc);
  constexpr int kMIter = (MH * MW + NT - 1) / NT;
  for (int k = 0; k < a.K; ++k) {
    // the weight sum of the M region (same for every frame; an L2 hit after
    // the first frame), loaded before waiting for the staged planes
    float nvr[kMIter];
#pragma unroll
    for (int j = 0; j < kMIter; ++j) {
      const int i = threadIdx.x + j * NT;
      const int X = x0 - 2 + i % MW, Y = y0 - 2 + i / MW;
      nvr[j] = (i < MH * MW && X >= 0 && Y >= 0 && X < a.wl && Y < a.hl) ? __ldg(a.norm + (int64_t)Y * a.pitch_l + X)
                                                                           : 0.0f;
    }
    cp_async_wait_all();
    __syncthreads();
    for (int i = threadIdx.x; i < GH * GW; i += NT) {
      const uint32_t v = S0.rgba[(i / GW) * SW + i % GW];
      S.gs[i] = make_float4(chf(v, 0), chf(v, 1), chf(v, 2), px_alpha(v) > 0 ? 1.0f : 0.0f);
    }
#pragma unroll
    for (int j = 0; j < kMIter; ++j) {
      const int i = threadIdx.x + j * NT;
      if (i >= MH * MW) break;
      const int X = x0 - 2 + i % MW, Y = y0 - 2 + i / MW;
      float m = 0.0f;
      if (X >= 0 && Y >= 0 && X < a.wl && Y < a.hl) {
        const float nv = nvr[j];
        m = nv > 1e-12f ? __fdiv_rn(S0.w[(i / MW) * SW + i % MW + 2], nv) : a.inv_count;
      }
      S.m[i] = m;
    }
    __syncthreads();
    if (k + 1 < a.K) stage_level0(S0, a, a.in0[k + 1], x0, y0);
    if (a.levels == 1) {
      // 1x1 image: the top level is level 0 (src/fuse/pyramid.zig:1605-1649)
#pragma unroll
      for (int i = 0; i < PPT; ++i) {
        const int p = acc_pixel(i);
        const int xx = p % TW, yy = p / TW;
        if (x0 + xx >= a.wl || y0 + yy >= a.hl) continue;
        const float m = S.m[(yy + 2) * MW + (xx + 2)];
        const float4 g = S.gs[(yy + 4) * GW + (xx + 4)];
        acc[i][0] = __fadd_rn(acc[i][0], __fmul_rn(g.x, m));
        acc[i][1] = __fadd_rn(acc[i][1], __fmul_rn(g.y, m));
        acc[i][2] = __fadd_rn(acc[i][2], __fmul_rn(g.z, m));
      }
      __syncthreads();
      continue;
    }
    reduce_step(S, a, x0, y0);
    store_next<T>(S, a, x0, y0, k);
    expand_blend_step(S, a, x0, y0, acc);
  }
  cp_async_wait_all();
  store_acc(a, x0, y0, acc);
}

// Level l -> l + 1 (l >= 1) for a batch of frames from their level planes.
template <typename T>
__global__ void __launch_bounds__(NT) level_kernel(const __grid_constant__ LevelArgs a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  LevelSmem& S = *reinterpret_cast<LevelSmem*>(smem_raw);
  const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  load_mask_support(S, a, x0, y0);
  float acc[PPT][3];
  // frame-parallel: this CTA blends frame blockIdx.z alone, from zero
  const int kb = a.frame_parallel ? (int)blockIdx.z : 0, ke = a.frame_parallel ? kb + 1 : a.K;
  if (a.frame_parallel) {
#pragma unroll
    for (int i = 0; i < PPT; ++i) acc[i][0] = acc[i][1] = acc[i][2] = 0.0f;
  } else {
    load_acc(a, x0, y0, acc);
  }
  for (int k = kb; k < ke; ++k) {
    const LevelPlanes& in = a.in[k];
    const T* g = (const T*)in.g;
    const T* mm = (const T*)in.m;
    for (int i = threadIdx.x; i < GH * GW; i += NT) {
      const int X = x0 - 4 + i % GW, Y = y0 - 4 + i / GW;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (X >= 0 && Y >= 0 && X < a.wl && Y < a.hl) {
        const int64_t o = (int64_t)Y * a.pitch_l + X;
        v = make_float4(ldv<T>(g, o), ldv<T>(g, in.plane + o), ldv<T>(g, 2 * in.plane + o), in.s[o] ? 1.0f : 0.0f);
      }
      S.gs[i] = v;
    }
    for (int i = threadIdx.x; i < MH * MW; i += NT) {
      const int X = x0 - 2 + i % MW, Y = y0 - 2 + i / MW;
      const bool inb = X >= 0 && Y >= 0 && X < a.wl && Y < a.hl;
      S.m[i] = inb ? ldv<T>(mm, (int64_t)Y * a.pitch_l + X) : 0.0f;
    }
    __syncthreads();
    reduce_step(S, a, x0, y0);
    store_next<T>(S, a, x0, y0, k);
    expand_blend_step(S, a, x0, y0, acc);
  }
  if (a.frame_parallel) {
    // 0 + (lap * m) is the product itself, so the ordered sum below adds
    // exactly the terms the sequential loop adds
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      const int p = acc_pixel(i);
      const int X = x0 + p % TW, Y = y0 + p / TW;
      if (X < a.wl && Y < a.hl) {
        const int64_t o = (int64_t)Y * a.pitch_l + X;
#pragma unroll
        for (int c = 0; c < 3; ++c) a.contrib[(int64_t)(kb * 3 + c) * a.acc_plane_l + o] = acc[i][c];
      }
    }
  } else {
    store_acc(a, x0, y0, acc);
  }
}

// ================================================== split pyramid kernels
// The image half (pass 1, as the frames arrive) and the mask half (pass 2,
// once the weight sum is complete) of a level step, with the Laplacians in
// HBM between them.  Every operation is the one of the fused kernels above,
// in the same order, so both give identical accumulators.
namespace {

struct __align__(16) ImgSmem {
  float4 gs[GH * GW];
  float tmp[kTmpFloats];
  float ng[3][NH * NW];
  uint8_t ns[NH * NW];
};
static_assert(offsetof(ImgSmem, tmp) % 16 == 0, "tmp is accessed as float4");

template <typename T>
__device__ void store_next_image(const ImgSmem& S, const LevelArgs& a, int x0, int y0, int k) {
  const int x1 = x0 >> 1, y1 = y0 >> 1;
  const bool top = a.level + 1 == a.levels - 1;
  for (int i = threadIdx.x; i < TH1 * TW1; i += NT) {
    const int ii = i / TW1, jj = i % TW1;
    const int xj = x1 + jj, yi = y1 + ii;
    if (xj >= a.wn || yi >= a.hn) continue;
    const int ni = (ii + 1) * NW + (jj + 1);
    const int64_t o = (int64_t)yi * a.pitch_n + xj;
    if (top) {
#pragma unroll
      for (int c = 0; c < 3; ++c) a.gtop[k][c * a.acc_plane_n + o] = S.ng[c][ni];
    } else {
      const LevelPlanes& out = a.out[k];
#pragma unroll
      for (int c = 0; c < 3; ++c) stv<T>((T*)out.g, c * out.plane + o, S.ng[c][ni]);
      out.s[o] = S.ns[ni];
    }
  }
}

}  // namespace

// One 64x32 tile of frame k's level step l -> l + 1 (the split pyramid's
// image half): Gaussian REDUCE, its store, and the tile's Laplacian.
template <typename T, bool L0>
__device__ __forceinline__ void img_tile(ImgSmem& S, const LevelArgs& a, int x0, int y0, int k) {
  // region loads issued together (all in flight before the first store)
  constexpr int NI = (GH * GW + NT - 1) / NT, HALF = (NI + 1) / 2;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float4 v[HALF];
#pragma unroll
    for (int j = 0; j < HALF; ++j) {
      const int i = threadIdx.x + (h * HALF + j) * NT;
      const int X = x0 - 4 + i % GW, Y = y0 - 4 + i / GW;
      v[j] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (i < GH * GW && X >= 0 && Y >= 0 && X < a.wl && Y < a.hl) {
        const int64_t o = (int64_t)Y * a.pitch_l + X;
        if constexpr (L0) {
          const uint32_t q = __ldg(a.in0[k].rgba + o);
          v[j] = make_float4(__uint_as_float(q), 0.f, 0.f, 0.f);
        } else {
          const LevelPlanes& in = a.in[k];
          const T* g = (const T*)in.g;
          v[j] = make_float4(ldv<T>(g, o), ldv<T>(g, in.plane + o), ldv<T>(g, 2 * in.plane + o),
                             in.s[o] ? 1.0f : 0.0f);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < HALF; ++j) {
      const int i = threadIdx.x + (h * HALF + j) * NT;
      if (i >= GH * GW) continue;
      if constexpr (L0) {
        const uint32_t q = __float_as_uint(v[j].x);
        S.gs[i] = make_float4(chf(q, 0), chf(q, 1), chf(q, 2), px_alpha(q) > 0 ? 1.0f : 0.0f);
      } else {
        S.gs[i] = v[j];
      }
    }
  }
  __syncthreads();
  reduce_image_step(S, a, x0, y0);
  store_next_image<T>(S, a, x0, y0, k);
  float unused[PPT][3];
  // the level-0 Laplacian stays FP32; the levels above are in the storage type
  using TL = typename std::conditional<L0, float, T>::type;
  expand_blend_step<true, ImgSmem, TL>(S, a, x0, y0, unused, (TL*)a.lap[k]);
}

template <typename T, bool L0>
__global__ void __launch_bounds__(NT) img_kernel(const __grid_constant__ LevelArgs a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  ImgSmem& S = *reinterpret_cast<ImgSmem*>(smem_raw);
  img_tile<T, L0>(S, a, blockIdx.x * TW, blockIdx.y * TH, blockIdx.z);
}

// Level-0 blend and level-0 mask REDUCE of a split-pyramid stack in one pass
// over each frame's weight and Laplacian.  A CTA owns a 64 x 32 level-0 tile
// (the 32 x 16 level-1 masks it REDUCEs to) and walks the frames in order.
// Per frame, each thread forms the normalised masks m = w / N (inv_count
// where N <= 1e-12; normalizeWeightsInto, src/fuse/pyramid.zig:303-316) of
// its two 4-pixel chunks, adds lap x m into its accumulators (the products
// and sums of the per-batch level-0 kernel, frame order) and stores
// m, zero where the union support is 0 or outside the level, into a shared
// region that adds the REDUCE halo (level-0 rows y0 - 2 .. y0 + 32, columns
// x0 - 4 .. x0 + 67 in 16-byte chunks; the halo's chunks are formed by the
// first threads).  After one barrier each thread REDUCEs two level-1 masks
// from the region with mask_reduce_kernel's five-tap sums in its order; the
// weight sums depend on the support alone and are formed once.  The region
// is double-buffered (one barrier per frame).  Each thread stages its own
// chunks of the next frame (weights, Laplacians, its halo weight) into shared
// memory with cp.async while the current frame is processed: only the thread
// that copies a chunk reads it, so the staging needs no barrier of its own,
// and a frame's loads have a whole frame's work to land in.  (Loads held in
// registers would cover only the REDUCE and leave 2 CTAs per SM waiting on
// HBM: 0.6 of the copy bandwidth against 0.77.)  No level-0 mask goes
// through HBM: per frame
// the weight (4 B) and the Laplacian (12 B) are read once and the level-1
// mask is written.
namespace {
constexpr int kB0Rows = kTileH + 3;                   // region rows: level-0 rows y0 - 2 .. y0 + 32
constexpr int kB0Chunks = kTileW / 4 + 2;             // 16-byte chunks per region row (x0 - 4 .. x0 + 67)
constexpr int kB0Stride = 4 * kB0Chunks;              // floats per region row
constexpr int kB0Halo = 3 * kB0Chunks + 2 * kTileH;   // rows 0, 1 and 34 whole, chunks 0 and 17 of the rest
static_assert(kThreads == 16 * (kTileH / 2) && kB0Halo <= kThreads, "two own chunks and at most one halo chunk per thread");

struct B0Chunk {
  int64_t off;      // element offset of the chunk in the level-0 planes
  float n[4];       // weight sums
  uint32_t keep;    // bit e: column e of the chunk is inside the level with union support
  int32_t so;       // offset of the chunk in the region (floats)
  bool in;          // the chunk's first column is inside the level (the chunk is read)
};

__device__ __forceinline__ B0Chunk b0_chunk(const float* norm, const uint8_t* sm, int64_t pitch, int wl, int hl,
                                            int x0, int y0, int rr, int cc, bool live = true) {
  B0Chunk c;
  const int Y = y0 - 2 + rr, X = x0 - 4 + 4 * cc;
  c.so = rr * kB0Stride + 4 * cc;
  c.keep = 0u;
  c.off = 0;
  c.in = false;
#pragma unroll
  for (int e = 0; e < 4; ++e) c.n[e] = 1.0f;
  if (live && Y >= 0 && Y < hl && X >= 0 && X < wl) {  // the chunk lies inside the row's pitch
    const int64_t o = (int64_t)Y * pitch + X;
    c.off = o;
    c.in = true;
    if (norm) {
      const float4 q = __ldg(reinterpret_cast<const float4*>(norm + o));
      c.n[0] = q.x; c.n[1] = q.y; c.n[2] = q.z; c.n[3] = q.w;
    }
    const uint32_t s = __ldg(reinterpret_cast<const uint32_t*>(sm + o));
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (X + e < wl && ((s >> (8 * e)) & 255u)) c.keep |= 1u << e;
  }
  return c;
}

// Correctly rounded a / b from y = RN(1 / b), the weight sum's reciprocal
// formed once per pixel: Markstein's division refinement (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990): q0 = RN(a y), then two steps
// q += (a - b q) y with exact FMA residuals; the first makes q faithful,
// and from a faithful quotient and the correctly rounded reciprocal the
// second rounds a / b correctly.  Five instructions per frame-pixel instead
// of an IEEE division; checked bit for bit against __fdiv_rn on 10^10 pairs
// of the normalisation's ranges (w in [2^-20, 2) and 0, b in [1e-12, 512],
// divisors with all-ones or zero significands among them).
__device__ __forceinline__ float div_by_rcp(float a, float b, float y) {
  const float q0 = __fmul_rn(a, y);
  const float q1 = __fmaf_rn(__fmaf_rn(-b, q0, a), y, q0);
  return __fmaf_rn(__fmaf_rn(-b, q1, a), y, q1);
}

// out[i] = w[i] / n[i] by div_by_rcp, for the check of its rounding.
__global__ void normalise_check_kernel(const float* w, const float* n, float* out, size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    out[i] = div_by_rcp(w[i], n[i], __frcp_rn(n[i]));
}

// w / N (inv_count where N <= 1e-12), N's reciprocals in ry.
__device__ __forceinline__ float4 b0_mask(const B0Chunk& c, const float (&ry)[4], float4 w, float inv_count) {
  float4 m;
  m.x = c.n[0] > 1e-12f ? div_by_rcp(w.x, c.n[0], ry[0]) : inv_count;
  m.y = c.n[1] > 1e-12f ? div_by_rcp(w.y, c.n[1], ry[1]) : inv_count;
  m.z = c.n[2] > 1e-12f ? div_by_rcp(w.z, c.n[2], ry[2]) : inv_count;
  m.w = c.n[3] > 1e-12f ? div_by_rcp(w.w, c.n[3], ry[3]) : inv_count;
  return m;
}

__device__ __forceinline__ float4 b0_keep(const B0Chunk& c, float4 m) {
  return make_float4((c.keep & 1u) ? m.x : 0.0f, (c.keep & 2u) ? m.y : 0.0f, (c.keep & 4u) ? m.z : 0.0f,
                     (c.keep & 8u) ? m.w : 0.0f);
}

// A chunk of four samples in storage TS into a 16-byte staging slot (16-bit
// samples fill its first 8 bytes), and back as four floats.
template <typename TS>
__device__ __forceinline__ void b0_copy(float4* dst, const TS* src, bool ok) {
  if constexpr (sizeof(TS) == 4) {
    cp_async16(dst, src, ok ? 16 : 0);
  } else {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 8 : 0) : "memory");
  }
}
template <typename TS>
__device__ __forceinline__ float4 b0_load(const float4* p) {
  if constexpr (sizeof(TS) == 4) {
    return *p;
  } else {
    const uint2 q = *reinterpret_cast<const uint2*>(p);
    const TS* h = reinterpret_cast<const TS*>(&q);
    return make_float4(ldv<TS>(h, 0), ldv<TS>(h, 1), ldv<TS>(h, 2), ldv<TS>(h, 3));
  }
}
}  // namespace

// cp.async.wait_group 1: all but the most recent group of this thread's
// asynchronous copies have landed.
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Dynamic shared memory: the double-buffered mask region, then the staged
// chunks of two frames, [stage][slot][thread] (slots: weight of the two own
// chunks, their Laplacian planes, the halo weight).
constexpr int kB0Slots = 9;
constexpr size_t kB0Smem = 2 * kB0Rows * kB0Stride * sizeof(float) + 2 * kB0Slots * kThreads * sizeof(float4);

// TS: storage of the level's Laplacians and masks; NORM: level 0, the
// masks formed from the weights (w / N) rather than read.
template <typename TS, typename TO, bool NORM>
__global__ void __launch_bounds__(kThreads, 2)
    blend0_reduce_kernel(float* acc, int64_t plane, int64_t pitch, int wl, int hl, const float* norm,
           const uint8_t* sm, const void* const* lap, const void* const* wgt, void* const* mask1,
           int64_t pitch_n, int wn, int hn, int frames, float inv_count) {
  extern __shared__ __align__(16) float b0_smem[];
  float* const reg0 = b0_smem;  // [2][kB0Rows * kB0Stride]
  float4* const stage = reinterpret_cast<float4*>(b0_smem + 2 * kB0Rows * kB0Stride);
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * kTileH;
  const int g = tid % 16, r = tid / 16;
  if (!NORM) norm = nullptr;
  const B0Chunk c0 = b0_chunk(norm, sm, pitch, wl, hl, x0, y0, 2 + r, 1 + g);
  const B0Chunk c1 = b0_chunk(norm, sm, pitch, wl, hl, x0, y0, 18 + r, 1 + g);
  int hr = 0, hc = 0;
  if (tid < 3 * kB0Chunks) {
    hr = tid < 2 * kB0Chunks ? tid / kB0Chunks : kB0Rows - 1;
    hc = tid % kB0Chunks;
  } else {
    const int q = tid - 3 * kB0Chunks;
    hr = 2 + q / 2;
    hc = (q & 1) ? kB0Chunks - 1 : 0;
  }
  const bool has_halo = tid < kB0Halo;
  const B0Chunk ch = b0_chunk(norm, sm, pitch, wl, hl, x0, y0, hr, hc, has_halo);
  // level 0: the weight sums' reciprocals, once for every frame
  float ry[3][4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    ry[0][e] = NORM ? __frcp_rn(c0.n[e]) : 0.0f;
    ry[1][e] = NORM ? __frcp_rn(c1.n[e]) : 0.0f;
    ry[2][e] = NORM ? __frcp_rn(ch.n[e]) : 0.0f;
  }
  const int ri = tid / 16, jp = tid % 16;
  const int I = y0 / 2 + ri, J = x0 / 2 + 2 * jp;
  const int tap0 = 2 * ri * kB0Stride + 4 * jp + 2;
  int ws0 = 0, ws1 = 0;
#pragma unroll
  for (int ky = 0; ky < 5; ++ky) {
    const int Y = 2 * I - 2 + ky;
    int h0 = 0, h1 = 0;
    if (Y >= 0 && Y < hl) {
      const uint8_t* srow = sm + (int64_t)Y * pitch;
#pragma unroll
      for (int u = 0; u < 7; ++u) {
        const int X = 2 * J - 2 + u;
        const int s = (X >= 0 && X < wl && __ldg(srow + X)) ? 1 : 0;
        if (u < 5) h0 += s * (int)kw(u);
        if (u >= 2) h1 += s * (int)kw(u - 2);
      }
    }
    ws0 += (int)kw(ky) * h0;
    ws1 += (int)kw(ky) * h1;
  }
  const float rws0 = ws0 > 0 ? __fdividef(1.0f, (float)ws0) : 0.0f;
  const float rws1 = ws1 > 0 ? __fdividef(1.0f, (float)ws1) : 0.0f;
  const bool out_row = I < hn;
  float a[2][3][4];
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int e = 0; e < 4; ++e) a[u][c][e] = 0.0f;
  auto slot = [&](int s, int i) { return stage + (s * kB0Slots + i) * kThreads + tid; };
  const bool blending = lap != nullptr;  // null: the masks alone (FUSED level 0)
  auto issue = [&](int k) {
    const int s = k & 1;
    const TS* wk = (const TS*)wgt[k];
    b0_copy<TS>(slot(s, 0), wk + c0.off, c0.in);
    b0_copy<TS>(slot(s, 1), wk + c1.off, c1.in);
    if (blending) {
      const TS* lk = (const TS*)lap[k];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        b0_copy<TS>(slot(s, 2 + c), lk + c * plane + c0.off, c0.in);
        b0_copy<TS>(slot(s, 5 + c), lk + c * plane + c1.off, c1.in);
      }
    }
    if (has_halo) b0_copy<TS>(slot(s, 8), wk + ch.off, ch.in);
  };
  // level 0: the normalised mask; above: the stored mask
  auto mask = [&](const B0Chunk& c, const float4* p, int i) {
    const float4 v = b0_load<TS>(p);
    return NORM ? b0_mask(c, ry[i], v, inv_count) : v;
  };
  auto blend = [&](float (&av)[3][4], int s, int i0, float4 m) {
    const float mv[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float4 l = b0_load<TS>(slot(s, i0 + c));
      const float lv[4] = {l.x, l.y, l.z, l.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) av[c][e] = __fadd_rn(av[c][e], __fmul_rn(lv[e], mv[e]));
    }
  };
  issue(0);
  cp_async_commit();
  for (int k = 0; k < frames; ++k) {
    const int s = k & 1;
    float* const buf = reg0 + s * kB0Rows * kB0Stride;
    if (k + 1 < frames) issue(k + 1);
    cp_async_commit();
    cp_async_wait1();
    {
      const float4 m0 = mask(c0, slot(s, 0), 0), m1 = mask(c1, slot(s, 1), 1);
      if (blending) {
        blend(a[0], s, 2, m0);
        blend(a[1], s, 5, m1);
      }
      *reinterpret_cast<float4*>(buf + c0.so) = b0_keep(c0, m0);
      *reinterpret_cast<float4*>(buf + c1.so) = b0_keep(c1, m1);
      if (has_halo) *reinterpret_cast<float4*>(buf + ch.so) = b0_keep(ch, mask(ch, slot(s, 8), 2));
    }
    __syncthreads();
    float v0 = 0.f, v1 = 0.f;
#pragma unroll
    for (int ky = 0; ky < 5; ++ky) {
      const float* row = buf + tap0 + ky * kB0Stride;
      const float2 p = *reinterpret_cast<const float2*>(row);
      const float4 q = *reinterpret_cast<const float4*>(row + 2);
      const float t[7] = {p.x, p.y, q.x, q.y, q.z, q.w, row[6]};
      float h0 = 0.f, h1 = 0.f;
#pragma unroll
      for (int kx = 0; kx < 5; ++kx) {
        h0 = fmaf(kw(kx), t[kx], h0);
        h1 = fmaf(kw(kx), t[2 + kx], h1);
      }
      v0 = fmaf(kw(ky), h0, v0);
      v1 = fmaf(kw(ky), h1, v1);
    }
    if (out_row) {
      TO* orow = (TO*)mask1[k] + (int64_t)I * pitch_n;
      if (J < wn) stv<TO>(orow, J, ws0 > 0 ? v0 * rws0 : 0.f);
      if (J + 1 < wn) stv<TO>(orow, J + 1, ws1 > 0 ? v1 * rws1 : 0.f);
    }
  }
  cp_async_wait_all();
  auto store = [&](const B0Chunk& c, const float (&av)[3][4]) {
    if (!c.in) return;
    const int64_t o = c.off;
    const int X = x0 - 4 + (c.so % kB0Stride);
    if (X + 3 < wl) {
#pragma unroll
      for (int ci = 0; ci < 3; ++ci)
        *reinterpret_cast<float4*>(acc + ci * plane + o) = make_float4(av[ci][0], av[ci][1], av[ci][2], av[ci][3]);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (X + e < wl)
#pragma unroll
          for (int ci = 0; ci < 3; ++ci) acc[ci * plane + o + e] = av[ci][e];
    }
  };
  if (blending) {
    store(c0, a[0]);
    store(c1, a[1]);
  }
}

// Blend of one level over all frames in order, one pixel per thread (the
// products and sums of the per-batch kernels, from acc = 0).
template <typename T>
__global__ void blend_kernel(float* acc, int64_t plane, int64_t pitch, int w, int h, const void* const* lap,
                             const void* const* mask, int frames) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)w * h) return;
  const int64_t o = (i / w) * pitch + i % w;
  float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
  constexpr int U = 4;
  for (int k0 = 0; k0 < frames; k0 += U) {
    float l0[U], l1[U], l2[U], mv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (k0 + u < frames) {
        const T* lk = (const T*)lap[k0 + u];
        l0[u] = ldv<T>(lk, o);
        l1[u] = ldv<T>(lk, plane + o);
        l2[u] = ldv<T>(lk, 2 * plane + o);
        mv[u] = ldv<T>((const T*)mask[k0 + u], o);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (k0 + u < frames) {
        a0 = __fadd_rn(a0, __fmul_rn(l0[u], mv[u]));
        a1 = __fadd_rn(a1, __fmul_rn(l1[u], mv[u]));
        a2 = __fadd_rn(a2, __fmul_rn(l2[u], mv[u]));
      }
    }
  }
  acc[o] = a0;
  acc[plane + o] = a1;
  acc[2 * plane + o] = a2;
}

cudaError_t launch_blend(float* acc, int64_t plane, int64_t pitch, int w, int h, const void* const* lap,
                         const void* const* mask, int frames, int storage, cudaStream_t s) {
  const int64_t n = (int64_t)w * h;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  switch (storage) {
    case FS_STORAGE_F32: blend_kernel<float><<<blocks, 256, 0, s>>>(acc, plane, pitch, w, h, lap, mask, frames); break;
    case FS_STORAGE_F16: blend_kernel<__half><<<blocks, 256, 0, s>>>(acc, plane, pitch, w, h, lap, mask, frames); break;
    case FS_STORAGE_BF16:
      blend_kernel<__nv_bfloat16><<<blocks, 256, 0, s>>>(acc, plane, pitch, w, h, lap, mask, frames);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// Mask REDUCE, streaming: each thread owns two neighbouring level-(l+1)
// columns and a strip of kReduceRows rows, and slides a five-row window of
// horizontal sums down the level-l mask (two new rows per output row), with
// the taps of a row in one vector load plus its two edges.  The products and
// sums are reduce_mask_step's, in its order: per row
// v = sum_kx fma(s ? kw : 0, m, v), ws = sum_kx (s ? kw : 0); per column
// v = sum_ky fma(kw, v_row, v), ws likewise; mask = ws > 0 ? v * (1 / ws) : 0.
// Taps outside the level count as support 0 and value 0 (a row outside
// contributes 0 to both sums, as its five zero-support taps do there).
constexpr int kReduceRows = 8, kReduceWarps = 4;

template <typename T>
__device__ __forceinline__ void ld4(const T* p, float* v) {
  if constexpr (std::is_same<T, float>::value) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
  } else {
    const uint2 q = *reinterpret_cast<const uint2*>(p);
    const T* h = reinterpret_cast<const T*>(&q);
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = ldv<T>(h, u);
  }
}

template <typename T>
__device__ __forceinline__ void ld2(const T* p, float* v) {
  if constexpr (std::is_same<T, float>::value) {
    const float2 q = *reinterpret_cast<const float2*>(p);
    v[0] = q.x; v[1] = q.y;
  } else {
    const uint32_t q = *reinterpret_cast<const uint32_t*>(p);
    const T* h = reinterpret_cast<const T*>(&q);
    v[0] = ldv<T>(h, 0);
    v[1] = ldv<T>(h, 1);
  }
}

// Two consecutive samples, one vector store (8 bytes of f32, 4 of f16/bf16).
template <typename T>
__device__ __forceinline__ void st2(T* p, float v0, float v1) {
  if constexpr (std::is_same<T, float>::value) {
    *reinterpret_cast<float2*>(p) = make_float2(v0, v1);
  } else {
    T h[2];
    stv<T>(h, 0, v0);
    stv<T>(h, 1, v1);
    *reinterpret_cast<uint32_t*>(p) = *reinterpret_cast<const uint32_t*>(h);
  }
}

// Four consecutive samples, one vector store (16 bytes of f32, 8 of f16/bf16).
template <typename T>
__device__ __forceinline__ void st4(T* p, const float* v) {
  if constexpr (std::is_same<T, float>::value) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    T h[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) stv<T>(h, u, v[u]);
    *reinterpret_cast<uint2*>(p) = *reinterpret_cast<const uint2*>(h);
  }
}

// Horizontal sums of level-l row r for output columns j0, j0 + 1.
template <typename T>
__device__ __forceinline__ void reduce_row(const T* in, const uint8_t* sm, int64_t pitch, int wl, int hl, int r,
                                           int j0, float* v, float* ws) {
  float m[7];
  uint32_t s4 = 0u, s2 = 0u, s6 = 0u;  // support bytes of taps 2..5, 0..1 and 6
#pragma unroll
  for (int u = 0; u < 7; ++u) m[u] = 0.0f;
  const int c = 2 * j0;  // a multiple of 4: the vector loads are aligned
  if (r >= 0 && r < hl) {
    const T* row = in + (int64_t)r * pitch;
    const uint8_t* srow = sm + (int64_t)r * pitch;
    // columns c .. c + 3 lie inside the row's pitch (c < wl, pitch a multiple of 32)
    ld4<T>(row + c, m + 2);
    s4 = *reinterpret_cast<const uint32_t*>(srow + c);
    if (c > 0) {
      ld2<T>(row + c - 2, m);
      s2 = *reinterpret_cast<const uint16_t*>(srow + c - 2);
    }
    if (c + 4 < wl) {
      m[6] = ldv<T>(row, c + 4);
      s6 = srow[c + 4];
    }
  }
  if (c + 3 >= wl) s4 &= (1u << (8 * (wl - c))) - 1u;  // columns past the level: no support (wl - c in 1..3)
  // a tap without support adds nothing: fma(kw, 0, a) = a = fma(0, m, a), so
  // the value sums take the supported samples (zero elsewhere) with the
  // weights 1, 4, 6, 4, 1, and the weight sums (integers <= 16) come from
  // the support bytes as dot products
  const uint32_t nz0 = __vcmpne4(__byte_perm(s2, s4, 0x5410u), 0u);  // taps 0..3
  const uint32_t nz1 = __vcmpne4(s4, 0u);                            // taps 2..5
  float mp[7];
  mp[0] = (nz0 & 0x000000ffu) ? m[0] : 0.0f;
  mp[1] = (nz0 & 0x0000ff00u) ? m[1] : 0.0f;
#pragma unroll
  for (int u = 0; u < 4; ++u) mp[2 + u] = (nz1 & (0xffu << (8 * u))) ? m[2 + u] : 0.0f;
  mp[6] = s6 ? m[6] : 0.0f;
  constexpr uint32_t kW = 0x04060401u;
  const int w0 = (int)__dp4a(nz0 & kW, 0x01010101u, (nz1 >> 16) & 1u);
  const int w1 = (int)__dp4a(nz1 & kW, 0x01010101u, s6 ? 1u : 0u);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float a = 0.f;
#pragma unroll
    for (int kx = 0; kx < 5; ++kx) a = fmaf(kw(kx), mp[2 * h + kx], a);
    v[h] = a;
    ws[h] = __int_as_float(0x4B000000 | (h == 0 ? w0 : w1)) - 8388608.0f;  // exact
  }
}

// Grid: frames fastest (blockIdx.x), then column and row blocks, so that the
// CTAs resident together read the same region's support (and, at level 0,
// weight sum) through L2 instead of fetching it again for every frame.
template <typename TI, typename TO>
__global__ void __launch_bounds__(32 * kReduceWarps) mask_reduce_kernel(const __grid_constant__ MaskReduceArgs a) {
  const int j0 = 2 * (int)(blockIdx.y * 32 + threadIdx.x);
  const int i0 = (int)(blockIdx.z * kReduceWarps + threadIdx.y) * kReduceRows;
  if (j0 >= a.wn || i0 >= a.hn) return;  // no barriers below
  const int i1 = min(i0 + kReduceRows, a.hn);
  const TI* in = (const TI*)a.in[blockIdx.x];
  TO* out = (TO*)a.out[blockIdx.x];
  // window of horizontal sums: rows 2i - 2 .. 2i + 2 for output row i
  float hv[5][2], hw[5][2];
#pragma unroll
  for (int u = 0; u < 3; ++u)
    reduce_row<TI>(in, a.sm, a.pitch_l, a.wl, a.hl, 2 * i0 - 2 + u, j0, hv[u], hw[u]);
  for (int i = i0; i < i1; ++i) {
    reduce_row<TI>(in, a.sm, a.pitch_l, a.wl, a.hl, 2 * i + 1, j0, hv[3], hw[3]);
    reduce_row<TI>(in, a.sm, a.pitch_l, a.wl, a.hl, 2 * i + 2, j0, hv[4], hw[4]);
    TO* orow = out + (int64_t)i * a.pitch_n;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float v = 0.f, ws = 0.f;
#pragma unroll
      for (int ky = 0; ky < 5; ++ky) {
        v = fmaf(kw(ky), hv[ky][h], v);
        ws = fmaf(kw(ky), hw[ky][h], ws);
      }
      if (j0 + h < a.wn) stv<TO>(orow, j0 + h, ws > 0.f ? v * __fdividef(1.0f, ws) : 0.f);
    }
#pragma unroll
    for (int u = 0; u < 3; ++u) {
      hv[u][0] = hv[u + 2][0];
      hv[u][1] = hv[u + 2][1];
      hw[u][0] = hw[u + 2][0];
      hw[u][1] = hw[u + 2][1];
    }
  }
}

template <typename TI>
static cudaError_t launch_mask_reduce_in(const MaskReduceArgs& a, dim3 grid, dim3 block, int out_storage,
                                         cudaStream_t s) {
  switch (out_storage) {
    case FS_STORAGE_F32: mask_reduce_kernel<TI, float><<<grid, block, 0, s>>>(a); break;
    case FS_STORAGE_F16: mask_reduce_kernel<TI, __half><<<grid, block, 0, s>>>(a); break;
    case FS_STORAGE_BF16: mask_reduce_kernel<TI, __nv_bfloat16><<<grid, block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_mask_reduce(const MaskReduceArgs& a, int frames, int in_storage, int out_storage,
                               cudaStream_t s) {
  const dim3 block(32, kReduceWarps);
  const unsigned gx = (unsigned)((a.wn + 63) / 64);
  const unsigned gy = (unsigned)((a.hn + kReduceWarps * kReduceRows - 1) / (kReduceWarps * kReduceRows));
  if (frames <= 0 || gx > 65535u || gy > 65535u) return cudaErrorInvalidValue;
  const dim3 grid((unsigned)frames, gx, gy);
  switch (in_storage) {
    case FS_STORAGE_F32: return launch_mask_reduce_in<float>(a, grid, block, out_storage, s);
    case FS_STORAGE_F16: return launch_mask_reduce_in<__half>(a, grid, block, out_storage, s);
    case FS_STORAGE_BF16: return launch_mask_reduce_in<__nv_bfloat16>(a, grid, block, out_storage, s);
    default: return cudaErrorInvalidValue;
  }
}

// ------------------------------------------------ streaming image pyramid
// One frame's pyramid step l -> l + 1 for the levels whose EXPAND clamps
// (exact_expand == 0), without shared memory: each lane owns the level-(l+1)
// column pair J0 = 2p, J1 = 2p + 1 and the level-l columns c = 4p .. 4p + 3,
// and walks down a strip of level-(l+1) rows.  Horizontal REDUCE sums of
// level-l rows 2r - 2 .. 2r + 2, added up in tap order as they arrive, give
// level-(l+1) row r; the EXPAND's horizontal pass takes the neighbouring columns J0 - 1
// and J1 + 1 from the adjacent lanes (shuffles), so lanes 0 and 31 of a warp
// only feed their neighbours and kImgPairs lanes emit.  The Laplacian of
// level-l rows 2q, 2q + 1 is emitted once row q + 1 is known.  Products and
// sums are those of reduce_image_step and expand_blend_step (clamped mode),
// in their order.
constexpr int kImgWarps = 4, kImgPairs = 30;

// Horizontal REDUCE sums (v0, v1, v2, weight) of level-l row y (l >= 1) for
// the lane's two level-(l+1) columns.  A tap without support adds nothing
// (fma(w, 0, s) = s = fma(0, v, s)), so the value sums take the supported
// samples (zero elsewhere) with the weights 1, 4, 6, 4, 1, and the weight
// sums (integers <= 16) come from the support bytes as dot products; samples
// outside the level have no support.
template <typename T>
__device__ __forceinline__ void img_row(const LevelArgs& a, int k, int y, int c, bool live, float4 (&hs)[2]) {
  float v[3][7];
  uint32_t s4 = 0u, s2 = 0u, s6 = 0u;  // support bytes of taps 2..5, 0..1 and 6
#pragma unroll
  for (int ch = 0; ch < 3; ++ch)
#pragma unroll
    for (int u = 0; u < 7; ++u) v[ch][u] = 0.0f;
  if (live && y >= 0 && y < a.hl) {
    const int64_t ro = (int64_t)y * a.pitch_l;
    // columns c .. c + 3 lie inside the row's pitch (c < wl, pitch a multiple of 32)
    const LevelPlanes& in = a.in[k];
    const T* g = (const T*)in.g + ro;
    const uint8_t* sp = in.s + ro;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      const T* gc = g + ch * in.plane;
      ld4<T>(gc + c, v[ch] + 2);
      if (c > 0) ld2<T>(gc + c - 2, v[ch]);
      if (c + 4 < a.wl) v[ch][6] = ldv<T>(gc, c + 4);
    }
    s4 = *reinterpret_cast<const uint32_t*>(sp + c);
    if (c > 0) s2 = *reinterpret_cast<const uint16_t*>(sp + c - 2);
    if (c + 4 < a.wl) s6 = sp[c + 4];
    if (c + 3 >= a.wl) s4 &= (1u << (8 * (a.wl - c))) - 1u;  // columns past the level (wl - c in 1..3)
  }
  const uint32_t nz0 = __vcmpne4(__byte_perm(s2, s4, 0x5410u), 0u);  // taps 0..3
  const uint32_t nz1 = __vcmpne4(s4, 0u);                            // taps 2..5
  bool sup[7];
  sup[0] = (nz0 & 0x000000ffu) != 0u;
  sup[1] = (nz0 & 0x0000ff00u) != 0u;
#pragma unroll
  for (int u = 0; u < 4; ++u) sup[2 + u] = (nz1 & (0xffu << (8 * u))) != 0u;
  sup[6] = s6 != 0u;
  constexpr uint32_t kW = 0x04060401u;
  const int wsum[2] = {(int)__dp4a(nz0 & kW, 0x01010101u, (nz1 >> 16) & 1u),
                       (int)__dp4a(nz1 & kW, 0x01010101u, s6 ? 1u : 0u)};
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float acc[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      float sum = 0.f;
#pragma unroll
      for (int kx = 0; kx < 5; ++kx) sum = fmaf(kw(kx), sup[2 * h + kx] ? v[ch][2 * h + kx] : 0.0f, sum);
      acc[ch] = sum;
    }
    hs[h] = make_float4(acc[0], acc[1], acc[2], __int_as_float(0x4B000000 | wsum[h]) - 8388608.0f);
  }
}

// Level 0 in integers: the samples are bytes and the weights 1, 4, 6 (or 0
// without support), so every partial sum of the FP32 REDUCE is an integer
// below 2^16 and exact; the integer sums equal it bit for bit.  Horizontal
// sums of one row for the lane's two columns: the channel bytes of taps
// 0..3 gathered into one word each and dot-multiplied with the tap weights
// (zeroed where alpha is 0), plus tap 4.
__device__ __forceinline__ void sum_row_u8(const uint32_t (&wr)[7], int c, int wl, int4 (&hs)[2]) {
  uint32_t w[7];
#pragma unroll
  for (int u = 0; u < 7; ++u) w[u] = (u < 2 || u == 6 || c + u - 2 < wl) ? wr[u] : 0u;  // words past the level
  constexpr uint32_t kW = 0x04060401u;  // tap weights 1, 4, 6, 4 (tap 4: 1)
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t b0 = w[2 * h], b1 = w[2 * h + 1], b2 = w[2 * h + 2], b3 = w[2 * h + 3], b4 = w[2 * h + 4];
    const uint32_t al = __byte_perm(__byte_perm(b0, b1, 0x0073u), __byte_perm(b2, b3, 0x0073u), 0x5410u);
    const uint32_t wt = __vcmpne4(al, 0u) & kW;
    const bool s4 = (b4 >> 24) != 0u;
    int v[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      const uint32_t sel = (uint32_t)ch | ((uint32_t)(4 + ch) << 4);
      const uint32_t g = __byte_perm(__byte_perm(b0, b1, sel), __byte_perm(b2, b3, sel), 0x5410u);
      v[ch] = (int)__dp4a(g, wt, s4 ? (b4 >> (8 * ch)) & 0xffu : 0u);
    }
    hs[h] = make_int4(v[0], v[1], v[2], (int)__dp4a(wt, 0x01010101u, s4 ? 1u : 0u));
  }
}

// The words of level-0 row y under the lane's taps (columns c - 2 .. c + 4);
// only loads, so that the next rows can be fetched while this one is summed.
__device__ __forceinline__ void load_row_u8(const LevelArgs& a, int k, int y, int c, bool live, uint32_t (&w)[7]) {
#pragma unroll
  for (int u = 0; u < 7; ++u) w[u] = 0u;
  if (live && y >= 0 && y < a.hl) {
    const uint32_t* row = a.in0[k].rgba + (int64_t)y * a.pitch_l;
    const uint4 q4 = *reinterpret_cast<const uint4*>(row + c);  // inside the row's pitch
    w[2] = q4.x;
    w[3] = q4.y;
    w[4] = q4.z;
    w[5] = q4.w;
    if (c > 0) {
      const uint2 q2 = *reinterpret_cast<const uint2*>(row + c - 2);
      w[0] = q2.x;
      w[1] = q2.y;
    }
    if (c + 4 < a.wl) w[6] = row[c + 4];
  }
}

__device__ __forceinline__ void img_row_u8(const LevelArgs& a, int k, int y, int c, bool live, int4 (&hs)[2]) {
  uint32_t w[7];
  load_row_u8(a, k, y, c, live, w);
  sum_row_u8(w, c, a.wl, hs);
}

// One vertical REDUCE tap: v = fma(w, row, v) on value and weight sums
// (integer sums at level 0).
__device__ __forceinline__ float4 vtap(int w, float4 t, float4 v) {
  const float f = (float)w;
  return make_float4(fmaf(f, t.x, v.x), fmaf(f, t.y, v.y), fmaf(f, t.z, v.z), fmaf(f, t.w, v.w));
}
__device__ __forceinline__ int4 vtap(int w, int4 t, int4 v) {
  return make_int4(v.x + w * t.x, v.y + w * t.y, v.z + w * t.z, v.w + w * t.w);
}
template <class A> __device__ __forceinline__ A acc_zero();
template <> __device__ __forceinline__ float4 acc_zero<float4>() { return make_float4(0.f, 0.f, 0.f, 0.f); }
template <> __device__ __forceinline__ int4 acc_zero<int4>() { return make_int4(0, 0, 0, 0); }
// exact float of a non-negative integer below 2^23
__device__ __forceinline__ float small_int_float(int v) { return __int_as_float(0x4B000000 | v) - 8388608.0f; }
__device__ __forceinline__ float4 acc_float(float4 v) { return v; }
__device__ __forceinline__ float4 acc_float(int4 v) {
  return make_float4(small_int_float(v.x), small_int_float(v.y), small_int_float(v.z), small_int_float(v.w));
}
template <typename T, bool L0, class A>
__device__ __forceinline__ void row_sums(const LevelArgs& a, int k, int y, int c, bool live, A (&hs)[2]) {
  if constexpr (L0) img_row_u8(a, k, y, c, live, hs);
  else img_row<T>(a, k, y, c, live, hs);
}
__device__ __forceinline__ int kwi(int i) { return (i == 0 || i == 4) ? 1 : ((i == 1 || i == 3) ? 4 : 6); }

template <typename T, bool L0>
__global__ void __launch_bounds__(32 * kImgWarps) img_stream_kernel(const __grid_constant__ LevelArgs a, int rows) {
  const int lane = (int)threadIdx.x, k = (int)blockIdx.z;
  const int first = ((int)blockIdx.x * kImgWarps + (int)threadIdx.y) * kImgPairs;  // pair of lane 1
  if (2 * first >= a.wn) return;  // the whole warp: none of its pairs is in the level
  const int p = first + lane - 1;
  const int J0 = 2 * p, c = 4 * p;
  const bool live = p >= 0 && J0 < a.wn;
  const bool emit = live && lane >= 1 && lane <= kImgPairs;
  const bool j1in = J0 + 1 < a.wn, rin = J0 + 2 < a.wn;
  const int i0 = (int)blockIdx.y * rows;
  const int i1 = min(i0 + rows, a.hn);
  using Acc = typename std::conditional<L0, int4, float4>::type;
  const Acc zero = acc_zero<Acc>();
  // vertical REDUCE sums in tap order (level-l rows 2r - 2 .. 2r + 2 for
  // level-(l+1) row r): cur = row r with taps 0 .. 2, nxt = row r + 1 with
  // tap 0; the level-l rows 2r + 1, 2r + 2 complete cur, advance nxt and
  // start row r + 2
  Acc cur[2], nxt[2];
  float Hm2[3][4], Hm1[3][4], Hc[3][4];
#pragma unroll
  for (int ch = 0; ch < 3; ++ch)
#pragma unroll
    for (int u = 0; u < 4; ++u) Hm2[ch][u] = Hm1[ch][u] = 0.0f;
  int r = i0 > 0 ? i0 - 1 : 0;
  // level 0: the lane's four words of level-l rows 2r - 2, 2r - 1, 2r at the
  // top of step r (the Laplacian rows emitted at step r are the first two)
  uint4 ringR = make_uint4(0u, 0u, 0u, 0u), ringQ = ringR, ringP = ringR;
  {
    Acc t0[2], t1[2], t2[2];
    if constexpr (L0) {
      uint32_t w0[7], w1[7], w2[7];
      load_row_u8(a, k, 2 * r - 2, c, live, w0);
      load_row_u8(a, k, 2 * r - 1, c, live, w1);
      load_row_u8(a, k, 2 * r, c, live, w2);
      sum_row_u8(w0, c, a.wl, t0);
      sum_row_u8(w1, c, a.wl, t1);
      sum_row_u8(w2, c, a.wl, t2);
      ringR = make_uint4(w0[2], w0[3], w0[4], w0[5]);
      ringQ = make_uint4(w1[2], w1[3], w1[4], w1[5]);
      ringP = make_uint4(w2[2], w2[3], w2[4], w2[5]);
    } else {
      row_sums<T, L0>(a, k, 2 * r - 2, c, live, t0);
      row_sums<T, L0>(a, k, 2 * r - 1, c, live, t1);
      row_sums<T, L0>(a, k, 2 * r, c, live, t2);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      cur[h] = vtap(kwi(2), t2[h], vtap(kwi(1), t1[h], vtap(kwi(0), t0[h], zero)));
      nxt[h] = vtap(kwi(0), t2[h], zero);
    }
  }
  uint32_t n3[7], n4[7];  // level 0: the words of the next two rows, fetched one step ahead
  if constexpr (L0) {
    load_row_u8(a, k, 2 * r + 1, c, live, n3);
    load_row_u8(a, k, 2 * r + 2, c, live, n4);
  }
  for (; r <= i1; ++r) {
    float4 fin[2];
    uint4 c3 = make_uint4(0u, 0u, 0u, 0u), c4 = c3;  // level 0: words of rows 2r + 1, 2r + 2
    {
      Acc t3[2], t4[2];
      if constexpr (L0) {
        uint32_t w3[7], w4[7];
#pragma unroll
        for (int u = 0; u < 7; ++u) {
          w3[u] = n3[u];
          w4[u] = n4[u];
        }
        if (r < i1) {
          load_row_u8(a, k, 2 * r + 3, c, live, n3);
          load_row_u8(a, k, 2 * r + 4, c, live, n4);
        }
        sum_row_u8(w3, c, a.wl, t3);
        sum_row_u8(w4, c, a.wl, t4);
        c3 = make_uint4(w3[2], w3[3], w3[4], w3[5]);
        c4 = make_uint4(w4[2], w4[3], w4[4], w4[5]);
      } else {
        row_sums<T, L0>(a, k, 2 * r + 1, c, live, t3);
        row_sums<T, L0>(a, k, 2 * r + 2, c, live, t4);
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        fin[h] = acc_float(vtap(kwi(4), t4[h], vtap(kwi(3), t3[h], cur[h])));
        cur[h] = vtap(kwi(2), t4[h], vtap(kwi(1), t3[h], nxt[h]));
        nxt[h] = vtap(kwi(0), t4[h], zero);
      }
    }
    if (r < a.hn) {  // warp-uniform
      // REDUCE: level-(l+1) row r, columns J0, J0 + 1
      float g[2][3];
      bool sp[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const float ws = fin[h].w;
        sp[h] = live && J0 + h < a.wn && ws > 0.f;
        const float rc = sp[h] ? __fdividef(1.0f, ws) : 0.0f;
        g[h][0] = fin[h].x * rc;
        g[h][1] = fin[h].y * rc;
        g[h][2] = fin[h].z * rc;
      }
      if (emit && r >= i0 && r < i1) {
        const LevelPlanes& out = a.out[k];
        const int64_t o = (int64_t)r * a.pitch_n + J0;  // J0 even: the pair is one aligned vector
        if (j1in) {
#pragma unroll
          for (int ch = 0; ch < 3; ++ch) st2<T>((T*)out.g + ch * out.plane + o, g[0][ch], g[1][ch]);
          *reinterpret_cast<uint16_t*>(out.s + o) = (uint16_t)((sp[0] ? 1u : 0u) | (sp[1] ? 0x100u : 0u));
        } else {
#pragma unroll
          for (int ch = 0; ch < 3; ++ch) stv<T>((T*)out.g, ch * out.plane + o, g[0][ch]);
          out.s[o] = sp[0] ? 1 : 0;
        }
      }
      // horizontal EXPAND of row r onto columns c .. c + 3 (clamped)
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) {
        const float gA = g[0][ch], gB = j1in ? g[1][ch] : gA;
        float gL = __shfl_up_sync(0xffffffffu, gB, 1);
        const float gRn = __shfl_down_sync(0xffffffffu, gA, 1);
        if (p == 0) gL = gA;
        const float gR = rin ? gRn : gB;
        Hc[ch][0] = __fmul_rn(__fadd_rn(__fadd_rn(gL, __fmul_rn(6.0f, gA)), gB), 0.125f);
        Hc[ch][1] = __fmul_rn(__fadd_rn(gA, gB), 0.5f);
        Hc[ch][2] = __fmul_rn(__fadd_rn(__fadd_rn(gA, __fmul_rn(6.0f, gB)), gR), 0.125f);
        Hc[ch][3] = __fmul_rn(__fadd_rn(gB, gR), 0.5f);
      }
      if (r == 0) {  // row -1 clamps to row 0
#pragma unroll
        for (int ch = 0; ch < 3; ++ch)
#pragma unroll
          for (int u = 0; u < 4; ++u) Hm1[ch][u] = Hc[ch][u];
      }
    } else {  // row hn clamps to row hn - 1
#pragma unroll
      for (int ch = 0; ch < 3; ++ch)
#pragma unroll
        for (int u = 0; u < 4; ++u) Hc[ch][u] = Hm1[ch][u];
    }
    // Laplacian of level-l rows 2q, 2q + 1, q = r - 1
    if (emit && r >= i0 + 1) {
#pragma unroll
      for (int yy = 0; yy < 2; ++yy) {
        const int y = 2 * (r - 1) + yy;
        if (y >= a.hl) break;
        const int64_t ro = (int64_t)y * a.pitch_l;
        float gv[3][4];
        if constexpr (L0) {
          const uint4 q4 = yy == 0 ? ringR : ringQ;  // rows 2r - 2, 2r - 1
          const uint32_t w[4] = {q4.x, q4.y, q4.z, q4.w};
#pragma unroll
          for (int ch = 0; ch < 3; ++ch)
#pragma unroll
            for (int u = 0; u < 4; ++u) gv[ch][u] = chf(w[u], ch);
        } else {
          const LevelPlanes& in = a.in[k];
#pragma unroll
          for (int ch = 0; ch < 3; ++ch) ld4<T>((const T*)in.g + ch * in.plane + ro + c, gv[ch]);
        }
        using TL = typename std::conditional<L0, float, T>::type;  // level-0 Laplacians stay FP32
        TL* lp = (TL*)a.lap[k] + ro + c;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
          float lv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            // odd rows: the reference's (H + H) * 0.5, which is H exactly
            const float e = yy == 0
                ? __fmul_rn(__fadd_rn(__fadd_rn(Hm2[ch][u], __fmul_rn(6.0f, Hm1[ch][u])), Hc[ch][u]), 0.125f)
                : Hm1[ch][u];
            lv[u] = __fsub_rn(gv[ch][u], e);
          }
          TL* lc = lp + ch * a.acc_plane_l;
          if (c + 3 < a.wl) {
            st4<TL>(lc, lv);
          } else {
#pragma unroll
            for (int u = 0; u < 4; ++u)
              if (c + u < a.wl) stv<TL>(lc, u, lv[u]);
          }
        }
      }
    }
#pragma unroll
    for (int ch = 0; ch < 3; ++ch)
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        Hm2[ch][u] = Hm1[ch][u];
        Hm1[ch][u] = Hc[ch][u];
      }
    if constexpr (L0) {
      ringR = ringP;
      ringQ = c3;
      ringP = c4;
    }
  }
}

// The same image step for l >= 1 with each warp's level-l rows staged in
// shared memory: a ring of kStageRows rows per warp, filled by cp.async one
// step (two rows) ahead of the REDUCE and kept for the Laplacian of the rows
// two and three steps back, so that a step's loads land while the previous
// step computes and the Laplacian reads no row from HBM again (the streaming
// kernel above reads each row's taps when it needs them and waits on HBM).
// Lane L copies its own four columns of each plane and of the support, lane
// 0 also the four before them (its REDUCE taps c - 2, c - 1), lane 31 the
// four after; the taps of a row are read from the ring after the lane's
// copies have landed (cp.async.wait_group) and the warp has met
// (__syncwarp), and a slot is refilled only after the warp has met again.
// Products, sums and their order are those of img_stream_kernel<T, false>.
constexpr int kStageRows = 7;       // level-l rows 2r - 2 .. 2r + 4 at step r
constexpr int kStageCols = 4 * 34;  // chunk 0: before lane 0; 1 + L: lane L; 33: after lane 31

template <typename T>
struct __align__(16) StageRow {
  T g[3][kStageCols];
  uint8_t s[kStageCols];
};

template <int N>
__device__ __forceinline__ void cp_async_ca(void* dst, const void* src, bool full) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (N == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(full ? 16 : 0) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src), "n"(N), "r"(full ? N : 0)
                 : "memory");
}

template <typename T>
__device__ __forceinline__ void stage_row(StageRow<T>& R, const LevelPlanes& in, int64_t pitch, int wl, int hl,
                                          int y, int c, int lane) {
  const bool rin = y >= 0 && y < hl;
  const int64_t ro = rin ? (int64_t)y * pitch : 0;
  const T* g = (const T*)in.g;
  auto chunk = [&](int dst, int col) {  // columns col .. col + 3, inside the row's pitch when col < wl
    const bool ok = rin && col >= 0 && col < wl;
    const int64_t o = ok ? ro + col : 0;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) cp_async_ca<4 * sizeof(T)>(&R.g[ch][dst], g + ch * in.plane + o, ok);
    cp_async_ca<4>(&R.s[dst], in.s + o, ok);
  };
  chunk(4 + 4 * lane, c);
  if (lane == 0) chunk(0, c - 4);
  if (lane == 31) chunk(4 * 33, c + 4);
}

// img_row from a staged row: taps c - 2 .. c + 4 at ring columns 4L + 2 .. 4L + 8.
template <typename T>
__device__ __forceinline__ void staged_row_sums(const StageRow<T>& R, int lane, int c, int wl, float4 (&hs)[2]) {
  float v[3][7];
  const int b = 4 * lane + 2;
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    ld2<T>(&R.g[ch][b], v[ch]);
    ld4<T>(&R.g[ch][b + 2], v[ch] + 2);
    v[ch][6] = ldv<T>(&R.g[ch][b + 6], 0);
  }
  const uint32_t s2 = *reinterpret_cast<const uint16_t*>(&R.s[b]);
  uint32_t s4 = *reinterpret_cast<const uint32_t*>(&R.s[b + 2]);
  const uint32_t s6 = c + 4 < wl ? R.s[b + 6] : 0u;
  if (c + 3 >= wl) s4 &= c < wl ? (1u << (8 * (wl - c))) - 1u : 0u;  // columns past the level
  const uint32_t nz0 = __vcmpne4(__byte_perm(s2, s4, 0x5410u), 0u);  // taps 0..3
  const uint32_t nz1 = __vcmpne4(s4, 0u);                            // taps 2..5
  bool sup[7];
  sup[0] = (nz0 & 0x000000ffu) != 0u;
  sup[1] = (nz0 & 0x0000ff00u) != 0u;
#pragma unroll
  for (int u = 0; u < 4; ++u) sup[2 + u] = (nz1 & (0xffu << (8 * u))) != 0u;
  sup[6] = s6 != 0u;
  constexpr uint32_t kW = 0x04060401u;
  const int wsum[2] = {(int)__dp4a(nz0 & kW, 0x01010101u, (nz1 >> 16) & 1u),
                       (int)__dp4a(nz1 & kW, 0x01010101u, s6 ? 1u : 0u)};
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float acc[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      float sum = 0.f;
#pragma unroll
      for (int kx = 0; kx < 5; ++kx) sum = fmaf(kw(kx), sup[2 * h + kx] ? v[ch][2 * h + kx] : 0.0f, sum);
      acc[ch] = sum;
    }
    hs[h] = make_float4(acc[0], acc[1], acc[2], __int_as_float(0x4B000000 | wsum[h]) - 8388608.0f);
  }
}

template <typename T>
__global__ void __launch_bounds__(32 * kImgWarps) img_stage_kernel(const __grid_constant__ LevelArgs a, int rows) {
  extern __shared__ __align__(16) uint8_t stage_smem[];
  StageRow<T>* const ring = reinterpret_cast<StageRow<T>*>(stage_smem) + threadIdx.y * kStageRows;
  const int lane = (int)threadIdx.x, k = (int)blockIdx.z;
  const int first = ((int)blockIdx.x * kImgWarps + (int)threadIdx.y) * kImgPairs;  // pair of lane 1
  if (2 * first >= a.wn) return;  // the whole warp: none of its pairs is in the level
  const int p = first + lane - 1;
  const int J0 = 2 * p, c = 4 * p;
  const bool live = p >= 0 && J0 < a.wn;
  const bool emit = live && lane >= 1 && lane <= kImgPairs;
  const bool j1in = J0 + 1 < a.wn, rin = J0 + 2 < a.wn;
  const int i0 = (int)blockIdx.y * rows;
  const int i1 = min(i0 + rows, a.hn);
  const LevelPlanes& in = a.in[k];
  auto slot = [&](int y) -> StageRow<T>& { return ring[(y + 2 * kStageRows) % kStageRows]; };
  auto sums = [&](int y, float4 (&hs)[2]) {
    if (live) {
      staged_row_sums<T>(slot(y), lane, c, a.wl, hs);
    } else {
      hs[0] = hs[1] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 cur[2], nxt[2];
  float Hm2[3][4], Hm1[3][4], Hc[3][4];
#pragma unroll
  for (int ch = 0; ch < 3; ++ch)
#pragma unroll
    for (int u = 0; u < 4; ++u) Hm2[ch][u] = Hm1[ch][u] = 0.0f;
  int r = i0 > 0 ? i0 - 1 : 0;
  for (int y = 2 * r - 2; y <= 2 * r + 2; ++y) stage_row<T>(slot(y), in, a.pitch_l, a.wl, a.hl, y, c, lane);
  cp_async_commit();
  cp_async_wait_all();
  __syncwarp();
  {
    float4 t0[2], t1[2], t2[2];
    sums(2 * r - 2, t0);
    sums(2 * r - 1, t1);
    sums(2 * r, t2);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      cur[h] = vtap(kwi(2), t2[h], vtap(kwi(1), t1[h], vtap(kwi(0), t0[h], zero)));
      nxt[h] = vtap(kwi(0), t2[h], zero);
    }
  }
  for (; r <= i1; ++r) {
    __syncwarp();  // every lane is done with the rows whose slots are refilled now
    if (r < i1) {
      stage_row<T>(slot(2 * r + 3), in, a.pitch_l, a.wl, a.hl, 2 * r + 3, c, lane);
      stage_row<T>(slot(2 * r + 4), in, a.pitch_l, a.wl, a.hl, 2 * r + 4, c, lane);
    }
    cp_async_commit();
    cp_async_wait1();  // rows 2r + 1, 2r + 2
    __syncwarp();
    float4 fin[2];
    {
      float4 t3[2], t4[2];
      sums(2 * r + 1, t3);
      sums(2 * r + 2, t4);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        fin[h] = vtap(kwi(4), t4[h], vtap(kwi(3), t3[h], cur[h]));
        cur[h] = vtap(kwi(2), t4[h], vtap(kwi(1), t3[h], nxt[h]));
        nxt[h] = vtap(kwi(0), t4[h], zero);
      }
    }
    if (r < a.hn) {  // warp-uniform
      float g[2][3];
      bool sp[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const float ws = fin[h].w;
        sp[h] = live && J0 + h < a.wn && ws > 0.f;
        const float rc = sp[h] ? __fdividef(1.0f, ws) : 0.0f;
        g[h][0] = fin[h].x * rc;
        g[h][1] = fin[h].y * rc;
        g[h][2] = fin[h].z * rc;
      }
      if (emit && r >= i0 && r < i1) {
        const LevelPlanes& out = a.out[k];
        const int64_t o = (int64_t)r * a.pitch_n + J0;  // J0 even: the pair is one aligned vector
        if (j1in) {
#pragma unroll
          for (int ch = 0; ch < 3; ++ch) st2<T>((T*)out.g + ch * out.plane + o, g[0][ch], g[1][ch]);
          *reinterpret_cast<uint16_t*>(out.s + o) = (uint16_t)((sp[0] ? 1u : 0u) | (sp[1] ? 0x100u : 0u));
        } else {
#pragma unroll
          for (int ch = 0; ch < 3; ++ch) stv<T>((T*)out.g, ch * out.plane + o, g[0][ch]);
          out.s[o] = sp[0] ? 1 : 0;
        }
      }
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) {
        const float gA = g[0][ch], gB = j1in ? g[1][ch] : gA;
        float gL = __shfl_up_sync(0xffffffffu, gB, 1);
        const float gRn = __shfl_down_sync(0xffffffffu, gA, 1);
        if (p == 0) gL = gA;
        const float gR = rin ? gRn : gB;
        Hc[ch][0] = __fmul_rn(__fadd_rn(__fadd_rn(gL, __fmul_rn(6.0f, gA)), gB), 0.125f);
        Hc[ch][1] = __fmul_rn(__fadd_rn(gA, gB), 0.5f);
        Hc[ch][2] = __fmul_rn(__fadd_rn(__fadd_rn(gA, __fmul_rn(6.0f, gB)), gR), 0.125f);
        Hc[ch][3] = __fmul_rn(__fadd_rn(gB, gR), 0.5f);
      }
      if (r == 0) {  // row -1 clamps to row 0
#pragma unroll
        for (int ch = 0; ch < 3; ++ch)
#pragma unroll
          for (int u = 0; u < 4; ++u) Hm1[ch][u] = Hc[ch][u];
      }
    } else {  // row hn clamps to row hn - 1
#pragma unroll
      for (int ch = 0; ch < 3; ++ch)
#pragma unroll
        for (int u = 0; u < 4; ++u) Hc[ch][u] = Hm1[ch][u];
    }
    // Laplacian of level-l rows 2q, 2q + 1, q = r - 1 (both still in the ring)
    if (emit && r >= i0 + 1) {
#pragma unroll
      for (int yy = 0; yy < 2; ++yy) {
        const int y = 2 * (r - 1) + yy;
        if (y >= a.hl) break;
        const int64_t ro = (int64_t)y * a.pitch_l;
        const StageRow<T>& R = slot(y);
        float gv[3][4];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) ld4<T>(&R.g[ch][4 + 4 * lane], gv[ch]);
        T* lp = (T*)a.lap[k] + ro + c;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
          float lv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            // odd rows: the reference's (H + H) * 0.5, which is H exactly
            const float e = yy == 0
                ? __fmul_rn(__fadd_rn(__fadd_rn(Hm2[ch][u], __fmul_rn(6.0f, Hm1[ch][u])), Hc[ch][u]), 0.125f)
                : Hm1[ch][u];
            lv[u] = __fsub_rn(gv[ch][u], e);
          }
          T* lc = lp + ch * a.acc_plane_l;
          if (c + 3 < a.wl) {
            st4<T>(lc, lv);
          } else {
#pragma unroll
            for (int u = 0; u < 4; ++u)
              if (c + u < a.wl) stv<T>(lc, u, lv[u]);
          }
        }
      }
    }
#pragma unroll
    for (int ch = 0; ch < 3; ++ch)
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        Hm2[ch][u] = Hm1[ch][u];
        Hm1[ch][u] = Hc[ch][u];
      }
  }
  cp_async_wait_all();
}

// Resident CTAs of a kernel per SM on this device's SMs (queried once per
// device ordinal below 64 into the caller's cache, one cache per kernel:
// kernels of one signature share their pointer type).
using ResidentCache = std::atomic<int>[64][2];
template <class K>
static int resident_ctas(K kernel, int threads, size_t smem, ResidentCache& cache, int* sms) {
  int dev = 0;
  cudaGetDevice(&dev);
  const int d = dev >= 0 && dev < 64 ? dev : 0;
  int per = cache[d][0].load(std::memory_order_relaxed), n = cache[d][1].load(std::memory_order_relaxed);
  if (per <= 0 || n <= 0 || dev >= 64) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess || per < 1) per = 1;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
    cudaGetLastError();
    cache[d][0].store(per, std::memory_order_relaxed);
    cache[d][1].store(n, std::memory_order_relaxed);
  }
  *sms = n;
  return per;
}

// Rows per strip: the candidate with the least estimated time, counted as
// whole waves of resident CTAs times the level-l rows a strip reads
// (2 rows + 3 of its REDUCE window): short strips fill the last wave of a
// small level, long ones read fewer window rows twice.
template <typename T, bool L0>
static cudaError_t launch_img_stream(const LevelArgs& a, cudaStream_t s) {
  const int pairs = (a.wn + 1) / 2;
  const int warps = (pairs + kImgPairs - 1) / kImgPairs;
  const int bx = (warps + kImgWarps - 1) / kImgWarps;
  int sms = 148;
  static ResidentCache cache;
  const int per_sm = resident_ctas(img_stream_kernel<T, L0>, 32 * kImgWarps, 0, cache, &sms);
  const int64_t slots = (int64_t)per_sm * sms;
  int rows = 32;
  int64_t best = INT64_MAX;
  for (int r : {32, 28, 24, 20, 16, 12, 8}) {
    const int64_t ctas = (int64_t)bx * ((a.hn + r - 1) / r) * a.K;
    const int64_t cost = ((ctas + slots - 1) / slots) * (2 * r + 3);
    if (cost < best) {
      best = cost;
      rows = r;
    }
  }
  const dim3 grid((unsigned)bx, (unsigned)((a.hn + rows - 1) / rows), (unsigned)a.K);
  img_stream_kernel<T, L0><<<grid, dim3(32, kImgWarps), 0, s>>>(a, rows);
  return cudaGetLastError();
}

template <typename T>
static cudaError_t launch_img_stage(const LevelArgs& a, cudaStream_t s) {
  constexpr size_t smem = sizeof(StageRow<T>) * kStageRows * kImgWarps;
  static DeviceOnce configured;
  cudaError_t e = configure(img_stage_kernel<T>, smem, &configured);
  if (e != cudaSuccess) return e;
  const int pairs = (a.wn + 1) / 2;
  const int warps = (pairs + kImgPairs - 1) / kImgPairs;
  const int bx = (warps + kImgWarps - 1) / kImgWarps;
  int sms = 148;
  static ResidentCache cache;
  const int per_sm = resident_ctas(img_stage_kernel<T>, 32 * kImgWarps, smem, cache, &sms);
  const int64_t slots = (int64_t)per_sm * sms;
  int rows = 32;
  int64_t best = INT64_MAX;
  for (int r : {32, 28, 24, 20, 16, 12, 8}) {
    const int64_t ctas = (int64_t)bx * ((a.hn + r - 1) / r) * a.K;
    const int64_t cost = ((ctas + slots - 1) / slots) * (2 * r + 3);
    if (cost < best) {
      best = cost;
      rows = r;
    }
  }
  const dim3 grid((unsigned)bx, (unsigned)((a.hn + rows - 1) / rows), (unsigned)a.K);
  img_stage_kernel<T><<<grid, dim3(32, kImgWarps), smem, s>>>(a, rows);
  return cudaGetLastError();
}

template <typename TS, typename TO, bool NORM>
static cudaError_t launch_blend_reduce_t(float* acc, int64_t plane, int64_t pitch, int w, int h, const float* norm,
                                         const uint8_t* sm, const void* const* lap, const void* const* mask,
                                         void* const* mask_next, int64_t pitch_n, int wn, int hn, int frames,
                                         float inv_count, cudaStream_t s) {
  static DeviceOnce cfg;
  cudaError_t e = configure(blend0_reduce_kernel<TS, TO, NORM>, kB0Smem, &cfg);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)((w + kTileW - 1) / kTileW), (unsigned)((h + kTileH - 1) / kTileH));
  blend0_reduce_kernel<TS, TO, NORM><<<grid, kThreads, kB0Smem, s>>>(acc, plane, pitch, w, h, norm, sm, lap, mask,
                                                                      mask_next, pitch_n, wn, hn, frames, inv_count);
  return cudaGetLastError();
}

template <typename TS, bool NORM>
static cudaError_t launch_blend_reduce_o(int out_storage, float* acc, int64_t plane, int64_t pitch, int w, int h,
                                         const float* norm, const uint8_t* sm, const void* const* lap,
                                         const void* const* mask, void* const* mask_next, int64_t pitch_n, int wn,
                                         int hn, int frames, float inv_count, cudaStream_t s) {
  switch (out_storage) {
    case FS_STORAGE_F32:
      return launch_blend_reduce_t<TS, float, NORM>(acc, plane, pitch, w, h, norm, sm, lap, mask, mask_next, pitch_n,
                                                    wn, hn, frames, inv_count, s);
    case FS_STORAGE_F16:
      return launch_blend_reduce_t<TS, __half, NORM>(acc, plane, pitch, w, h, norm, sm, lap, mask, mask_next, pitch_n,
                                                     wn, hn, frames, inv_count, s);
    case FS_STORAGE_BF16:
      return launch_blend_reduce_t<TS, __nv_bfloat16, NORM>(acc, plane, pitch, w, h, norm, sm, lap, mask, mask_next,
                                                            pitch_n, wn, hn, frames, inv_count, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_normalise_check(const float* w, const float* n, float* out, size_t count, cudaStream_t s) {
  if (count == 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  normalise_check_kernel<<<(unsigned)(8 * sms), 256, 0, s>>>(w, n, out, count);
  return cudaGetLastError();
}

cudaError_t launch_blend0_reduce(float* acc, int64_t plane, int64_t pitch, int w, int h, const float* norm,
                                 const uint8_t* sm, const float* const* lap, const float* const* wgt,
                                 void* const* mask1, int64_t pitch_n, int wn, int hn, int frames, float inv_count,
                                 int out_storage, cudaStream_t s) {
  if (frames <= 0 || (h + kTileH - 1) / kTileH > 65535) return cudaErrorInvalidValue;
  return launch_blend_reduce_o<float, true>(out_storage, acc, plane, pitch, w, h, norm, sm,
                                            (const void* const*)lap, (const void* const*)wgt, mask1, pitch_n, wn, hn,
                                            frames, inv_count, s);
}

cudaError_t launch_blend_reduce(float* acc, int64_t plane, int64_t pitch, int w, int h, const uint8_t* sm,
                                const void* const* lap, const void* const* mask, void* const* mask_next,
                                int64_t pitch_n, int wn, int hn, int frames, int storage, int out_storage,
                                cudaStream_t s) {
  if (frames <= 0 || (h + kTileH - 1) / kTileH > 65535) return cudaErrorInvalidValue;
  switch (storage) {
    case FS_STORAGE_F32:
      return launch_blend_reduce_o<float, false>(out_storage, acc, plane, pitch, w, h, nullptr, sm, lap, mask,
                                                 mask_next, pitch_n, wn, hn, frames, 0.0f, s);
    case FS_STORAGE_F16:
      return launch_blend_reduce_o<__half, false>(out_storage, acc, plane, pitch, w, h, nullptr, sm, lap, mask,
                                                  mask_next, pitch_n, wn, hn, frames, 0.0f, s);
    case FS_STORAGE_BF16:
      return launch_blend_reduce_o<__nv_bfloat16, false>(out_storage, acc, plane, pitch, w, h, nullptr, sm, lap, mask,
                                                         mask_next, pitch_n, wn, hn, frames, 0.0f, s);
    default: return cudaErrorInvalidValue;
  }
}

template <template <typename, bool> class KER, bool L0>
static cudaError_t launch_split(const LevelArgs& a, int storage, cudaStream_t s, DeviceOnce* cfg) {
  dim3 grid((a.wl + TW - 1) / TW, (a.hl + TH - 1) / TH, a.K);
  const size_t sm = sizeof(ImgSmem);
  cudaError_t e;
  switch (storage) {
    case FS_STORAGE_F32:
      if ((e = configure(KER<float, L0>::kernel, sm, &cfg[0])) != cudaSuccess) return e;
      KER<float, L0>::kernel<<<grid, NT, sm, s>>>(a);
      break;
    case FS_STORAGE_F16:
      if ((e = configure(KER<__half, L0>::kernel, sm, &cfg[1])) != cudaSuccess) return e;
      KER<__half, L0>::kernel<<<grid, NT, sm, s>>>(a);
      break;
    case FS_STORAGE_BF16:
      if ((e = configure(KER<__nv_bfloat16, L0>::kernel, sm, &cfg[2])) != cudaSuccess) return e;
      KER<__nv_bfloat16, L0>::kernel<<<grid, NT, sm, s>>>(a);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
template <typename T, bool L0> struct ImgK {
  static constexpr auto kernel = img_kernel<T, L0>;
};

cudaError_t launch_img_level(const LevelArgs& a, int storage, cudaStream_t s) {
  static DeviceOnce cfg0[3], cfg1[3];
  // clamped-EXPAND levels (never followed by the top level): streaming kernel
  if (!a.exact_expand && a.level + 2 < a.levels) {
    switch (storage) {
      case FS_STORAGE_F32:
        return a.level == 0 ? launch_img_stream<float, true>(a, s) : launch_img_stage<float>(a, s);
      case FS_STORAGE_F16:
        return a.level == 0 ? launch_img_stream<__half, true>(a, s) : launch_img_stage<__half>(a, s);
      case FS_STORAGE_BF16:
        return a.level == 0 ? launch_img_stream<__nv_bfloat16, true>(a, s) : launch_img_stage<__nv_bfloat16>(a, s);
      default:
        return cudaErrorInvalidValue;
    }
  }
  return a.level == 0 ? launch_split<ImgK, true>(a, storage, s, cfg0)
                      : launch_split<ImgK, false>(a, storage, s, cfg1);
}


// ====================================================== small-level tail
// The split pyramid's levels whose sides are at most kTailSide (a handful of
// 64x32 tiles each, too small to fill the GPU) go through three launches per
// stack instead of four per level: every operation and its order are those
// of the per-level kernels (img_tile, mask_reduce_kernel's rows, blend_kernel,
// collapse_kernel's no-wrap EXPAND), so the bytes are the same.

// Pass 1: one frame per CTA walks the tail's level steps in order; a level's
// Gaussian written by this CTA is read back by it at the next level (after
// the barrier that ends img_tile).
template <typename T>
__global__ void __launch_bounds__(NT) img_tail_kernel(const __grid_constant__ ImgTailArgs t) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  ImgSmem& S = *reinterpret_cast<ImgSmem*>(smem_raw);
  const int k = blockIdx.x;
  for (int i = 0; i < t.steps; ++i) {
    const LevelArgs& a = t.lv[i];
    for (int y0 = 0; y0 < a.hl; y0 += TH)
      for (int x0 = 0; x0 < a.wl; x0 += TW) img_tile<T, false>(S, a, x0, y0, k);
  }
}

cudaError_t launch_img_tail(const ImgTailArgs& a, int frames, int storage, cudaStream_t s) {
  static DeviceOnce cfg[3];
  if (a.steps < 1 || a.steps > kMaxTail || frames < 1) return cudaErrorInvalidValue;
  const size_t sm = sizeof(ImgSmem);
  cudaError_t e;
  switch (storage) {
    case FS_STORAGE_F32:
      if ((e = configure(img_tail_kernel<float>, sm, &cfg[0])) != cudaSuccess) return e;
      img_tail_kernel<float><<<frames, NT, sm, s>>>(a);
      break;
    case FS_STORAGE_F16:
      if ((e = configure(img_tail_kernel<__half>, sm, &cfg[1])) != cudaSuccess) return e;
      img_tail_kernel<__half><<<frames, NT, sm, s>>>(a);
      break;
    case FS_STORAGE_BF16:
      if ((e = configure(img_tail_kernel<__nv_bfloat16>, sm, &cfg[2])) != cudaSuccess) return e;
      img_tail_kernel<__nv_bfloat16><<<frames, NT, sm, s>>>(a);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// Bytes of the tail's mask-support levels T+1 .. L-1 in shared memory (each
// at most 32 x 32 at its 32-element pitch, every later one at most half as
// tall).
constexpr int kTailSupportBytes = 4096;

// Pass 2, masks: frame blockIdx.x, levels T+1 .. L-1.  The support of level
// l + 1 is any supported in-range tap of the 5x5 window below it
// (mask_support_kernel); the mask REDUCE of each output pair is
// mask_reduce_kernel's: the five rows' horizontal sums (reduce_row), then the
// vertical taps in order.
template <typename TS>
__global__ void __launch_bounds__(NT) mask_tail_kernel(const __grid_constant__ BlendTailArgs a) {
  __shared__ __align__(16) uint8_t sms[kTailSupportBytes];
  const int k = blockIdx.x, N = a.frames, nlev = a.levels - a.first;
  const uint8_t* sup[kMaxTail + 1];
  sup[0] = a.sm_first;
  int off = 0;
  for (int i = 1; i < nlev; ++i) {
    const TailLevel& P = a.lv[i - 1];
    const TailLevel& C = a.lv[i];
    uint8_t* dst = sms + off;
    off += (int)(C.pitch * C.h + 15) & ~15;
    for (int p = threadIdx.x; p < C.w * C.h; p += NT) {
      const int x = p % C.w, y = p / C.w;
      uint8_t any = 0;
      for (int ky = 0; ky < 5 && !any; ++ky) {
        const int sy = 2 * y - 2 + ky;
        if (sy < 0 || sy >= P.h) continue;
        for (int kx = 0; kx < 5; ++kx) {
          const int sx = 2 * x - 2 + kx;
          if (sx < 0 || sx >= P.w) continue;
          if (sup[i - 1][(int64_t)sy * P.pitch + sx]) {
            any = 1;
            break;
          }
        }
      }
      dst[(int64_t)y * C.pitch + x] = any;
    }
    sup[i] = dst;
    __syncthreads();
  }
  for (int i = 0; i + 1 < nlev; ++i) {
    const int l = a.first + i;
    const TailLevel& P = a.lv[i];
    const TailLevel& C = a.lv[i + 1];
    const TS* in = (const TS*)a.tab[(size_t)l * 2 * N + N + k];
    void* out = const_cast<void*>(a.tab[(size_t)(l + 1) * 2 * N + N + k]);
    const bool top = l + 2 == a.levels;  // the top mask is f32
    const int pairs = (C.w + 1) / 2;
    for (int t = threadIdx.x; t < pairs * C.h; t += NT) {
      const int j0 = 2 * (t % pairs), r = t / pairs;
      float hv[5][2], hw[5][2];
#pragma unroll
      for (int u = 0; u < 5; ++u) reduce_row<TS>(in, sup[i], P.pitch, P.w, P.h, 2 * r - 2 + u, j0, hv[u], hw[u]);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float v = 0.f, ws = 0.f;
#pragma unroll
        for (int ky = 0; ky < 5; ++ky) {
          v = fmaf(kw(ky), hv[ky][h], v);
          ws = fmaf(kw(ky), hw[ky][h], ws);
        }
        if (j0 + h < C.w) {
          const float m = ws > 0.f ? v * __fdividef(1.0f, ws) : 0.f;
          const int64_t o = (int64_t)r * C.pitch + j0 + h;
          if (top) stv<float>((float*)out, o, m);
          else stv<TS>((TS*)out, o, m);
        }
      }
    }
    __syncthreads();
  }
}

// Horizontal no-wrap EXPAND of child row `row` at parent column x (zero
// outside the child), expand_h1's operations.
__device__ __forceinline__ float tail_expand_h(const float* row, int x, int wc) {
  const int j = x >> 1;
  auto g = [&](int i) { return (i < 0 || i >= wc) ? 0.0f : row[i]; };
  if (x & 1) return __fmul_rn(4.0f, __fadd_rn(g(j), g(j + 1)));
  return __fadd_rn(__fadd_rn(g(j - 1), __fmul_rn(6.0f, g(j))), g(j + 1));
}

// Shared-memory bytes of the tail's accumulators (3 planes per level, rows
// of the level's width).
__host__ __device__ inline int tail_acc_floats(const BlendTailArgs& a) {
  int n = 0;
  for (int i = 0; i < a.levels - a.first; ++i) n += 3 * a.lv[i].w * a.lv[i].h;
  return n;
}

// Pass 2, blend + collapse: one thread per pixel of the tail levels forms
// acc_l = sum over frames in order of lap * mask (blend_kernel, its loads
// issued four frames at a time); the last CTA to finish (a ticket on
// a.counter, no waiting) brings every tail level's accumulator into shared
// memory, adds EXPAND(acc_l) into acc_{l-1} from the top down to level T with
// collapse_kernel's no-wrap operations (every tail parent is at most
// kTailSide <= 512 wide), writes level T back and resets the ticket.
template <typename TS>
__global__ void __launch_bounds__(256) blend_tail_kernel(const __grid_constant__ BlendTailArgs a) {
  extern __shared__ float tsm[];
  __shared__ bool last;
  const int N = a.frames, nlev = a.levels - a.first;
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int i = 0;
  while (i < nlev && g >= (int64_t)a.lv[i].w * a.lv[i].h) {
    g -= (int64_t)a.lv[i].w * a.lv[i].h;
    ++i;
  }
  if (i < nlev) {
    const TailLevel& V = a.lv[i];
    const int l = a.first + i;
    const int64_t o = (g / V.w) * V.pitch + g % V.w;
    const void* const* lap = a.tab + (size_t)l * 2 * N;
    const void* const* msk = lap + N;
    const bool top = l + 1 == a.levels;  // the top level's Gaussians and masks are f32
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
    constexpr int U = 4;
    for (int f0 = 0; f0 < N; f0 += U) {
      float l0[U], l1[U], l2[U], mv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (f0 + u < N) {
          if (top) {
            const float* lk = (const float*)lap[f0 + u];
            l0[u] = lk[o];
            l1[u] = lk[V.plane + o];
            l2[u] = lk[2 * V.plane + o];
            mv[u] = ((const float*)msk[f0 + u])[o];
          } else {
            const TS* lk = (const TS*)lap[f0 + u];
            l0[u] = ldv<TS>(lk, o);
            l1[u] = ldv<TS>(lk, V.plane + o);
            l2[u] = ldv<TS>(lk, 2 * V.plane + o);
            mv[u] = ldv<TS>((const TS*)msk[f0 + u], o);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (f0 + u < N) {
          a0 = __fadd_rn(a0, __fmul_rn(l0[u], mv[u]));
          a1 = __fadd_rn(a1, __fmul_rn(l1[u], mv[u]));
          a2 = __fadd_rn(a2, __fmul_rn(l2[u], mv[u]));
        }
      }
    }
    V.acc[o] = a0;
    V.acc[V.plane + o] = a1;
    V.acc[2 * V.plane + o] = a2;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(a.counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the tail accumulators into shared memory: level i at off[i], plane c at
  // + c * w * h, rows of w floats
  int off[kMaxTail + 1];
  {
    int n = 0;
    for (int k = 0; k < nlev; ++k) {
      off[k] = n;
      const TailLevel& V = a.lv[k];
      for (int e = threadIdx.x; e < 3 * V.w * V.h; e += blockDim.x) {
        const int c = e / (V.w * V.h), r = e % (V.w * V.h);
        tsm[n + e] = __ldcg(V.acc + c * V.plane + (int64_t)(r / V.w) * V.pitch + r % V.w);
      }
      n += 3 * V.w * V.h;
    }
  }
  __syncthreads();
  for (int c_i = nlev - 1; c_i >= 1; --c_i) {
    const TailLevel& C = a.lv[c_i];
    const TailLevel& P = a.lv[c_i - 1];
    const float* cs = tsm + off[c_i];
    float* ps = tsm + off[c_i - 1];
    for (int p = threadIdx.x; p < P.w * P.h; p += blockDim.x) {
      const int x = p % P.w, y = p / P.w, q = y >> 1;
      const float div = exact_expand_divisor(x, y, C.w, C.h);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float* cp = cs + c * C.w * C.h;
        auto hrow = [&](int row) -> float {  // zero rows outside the child
          return (row < 0 || row >= C.h) ? 0.0f : tail_expand_h(cp + row * C.w, x, C.w);
        };
        float v;
        if (y & 1) v = __fadd_rn(hrow(q), hrow(q + 1));
        else v = __fadd_rn(__fadd_rn(hrow(q - 1), __fmul_rn(6.0f, hrow(q))), hrow(q + 1));
        float* dst = ps + c * P.w * P.h + p;
        *dst = __fadd_rn(*dst, __fdiv_rn(v, div));
      }
    }
    __syncthreads();
  }
  {
    const TailLevel& V = a.lv[0];
    for (int e = threadIdx.x; e < 3 * V.w * V.h; e += blockDim.x) {
      const int c = e / (V.w * V.h), r = e % (V.w * V.h);
      V.acc[c * V.plane + (int64_t)(r / V.w) * V.pitch + r % V.w] = tsm[e];
    }
  }
  if (threadIdx.x == 0) *a.counter = 0u;
}

cudaError_t launch_mask_tail(const BlendTailArgs& a, cudaStream_t s) {
  const int nlev = a.levels - a.first;
  if (a.first < 1 || nlev < 2 || nlev > kMaxTail + 1 || a.frames < 1) return cudaErrorInvalidValue;
  int bytes = 0;
  for (int i = 1; i < nlev; ++i) bytes += (int)(a.lv[i].pitch * a.lv[i].h + 15) & ~15;
  if (bytes > kTailSupportBytes) return cudaErrorInvalidValue;
  switch (a.storage) {
    case FS_STORAGE_F32: mask_tail_kernel<float><<<a.frames, NT, 0, s>>>(a); break;
    case FS_STORAGE_F16: mask_tail_kernel<__half><<<a.frames, NT, 0, s>>>(a); break;
    case FS_STORAGE_BF16: mask_tail_kernel<__nv_bfloat16><<<a.frames, NT, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// Largest shared memory of the blend tail: every level's side is at most
// kTailSide, so its accumulators take at most 3 x 4 x (64^2 + 32^2 + ...) B.
constexpr size_t kTailAccBytes = 3 * 4 * (kTailSide * kTailSide * 4 / 3 + 64);

cudaError_t launch_blend_tail(const BlendTailArgs& a, cudaStream_t s) {
  static DeviceOnce cfg[3];
  const int nlev = a.levels - a.first;
  if (a.first < 1 || nlev < 2 || nlev > kMaxTail + 1 || a.frames < 1 || !a.counter) return cudaErrorInvalidValue;
  int64_t px = 0;
  for (int i = 0; i < nlev; ++i) {
    if (a.lv[i].w > kTailSide || a.lv[i].h > kTailSide) return cudaErrorInvalidValue;
    px += (int64_t)a.lv[i].w * a.lv[i].h;
  }
  const size_t sm = (size_t)tail_acc_floats(a) * sizeof(float);
  if (sm > kTailAccBytes) return cudaErrorInvalidValue;
  const unsigned blocks = (unsigned)((px + 255) / 256);
  cudaError_t e;
  switch (a.storage) {
    case FS_STORAGE_F32:
      if ((e = configure(blend_tail_kernel<float>, kTailAccBytes, &cfg[0])) != cudaSuccess) return e;
      blend_tail_kernel<float><<<blocks, 256, sm, s>>>(a);
      break;
    case FS_STORAGE_F16:
      if ((e = configure(blend_tail_kernel<__half>, kTailAccBytes, &cfg[1])) != cudaSuccess) return e;
      blend_tail_kernel<__half><<<blocks, 256, sm, s>>>(a);
      break;
    case FS_STORAGE_BF16:
      if ((e = configure(blend_tail_kernel<__nv_bfloat16>, kTailAccBytes, &cfg[2])) != cudaSuccess) return e;
      blend_tail_kernel<__nv_bfloat16><<<blocks, 256, sm, s>>>(a);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

__global__ void sum_contrib_kernel(float* acc, int64_t plane, int64_t pitch, int w, int h, const float* contrib,
                                   int K) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)w * h) return;
  const int64_t o = (i / w) * pitch + i % w;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float v = acc[c * plane + o];
    for (int k = 0; k < K; ++k) v = __fadd_rn(v, contrib[(int64_t)(k * 3 + c) * plane + o]);
    acc[c * plane + o] = v;
  }
}

cudaError_t launch_sum_contrib(float* acc, int64_t plane, int64_t pitch, int w, int h, const float* contrib, int K,
                               cudaStream_t s) {
  const int64_t n = (int64_t)w * h;
  sum_contrib_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(acc, plane, pitch, w, h, contrib, K);
  return cudaGetLastError();
}


template <template <typename> class KER>
static cudaError_t launch_levels(const LevelArgs& a, int storage, cudaStream_t s, DeviceOnce* cfg) {
  const size_t sm = KER<float>::smem();
  dim3 grid((a.wl + TW - 1) / TW, (a.hl + TH - 1) / TH, a.frame_parallel ? a.K : 1);
  cudaError_t e;
  switch (storage) {
    case FS_STORAGE_F32:
      if ((e = configure(KER<float>::fn(), sm, &cfg[0])) != cudaSuccess) return e;
      KER<float>::fn()<<<grid, NT, sm, s>>>(a);
      break;
    case FS_STORAGE_F16:
      if ((e = configure(KER<__half>::fn(), sm, &cfg[1])) != cudaSuccess) return e;
      KER<__half>::fn()<<<grid, NT, sm, s>>>(a);
      break;
    case FS_STORAGE_BF16:
      if ((e = configure(KER<__nv_bfloat16>::fn(), sm, &cfg[2])) != cudaSuccess) return e;
      KER<__nv_bfloat16>::fn()<<<grid, NT, sm, s>>>(a);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
template <typename T> struct Level0K {
  static decltype(&level0_kernel<T>) fn() { return &level0_kernel<T>; }
  static size_t smem() { return sizeof(Level0Smem); }
};
template <typename T> struct LevelK {
  static decltype(&level_kernel<T>) fn() { return &level_kernel<T>; }
  static size_t smem() { return sizeof(LevelSmem); }
};

cudaError_t launch_level0(const LevelArgs& a, int storage, cudaStream_t s) {
  static DeviceOnce cfg[3];
  return launch_levels<Level0K>(a, storage, s, cfg);
}

cudaError_t launch_level(const LevelArgs& a, int storage, cudaStream_t s) {
  static DeviceOnce cfg[3];
  return launch_levels<LevelK>(a, storage, s, cfg);
}

// ============================================== fused pass 1 (LAPS mode)
// One kernel for the level-0 part of a frame's pyramid, as the frames
// arrive: remap the 64x32 tile plus halo into shared memory, local-contrast
// weight w (added to the weight sum and union as in remap_weights_kernel),
// support-aware REDUCE of the remapped tile to the level-1 Gaussian (exact
// integer sums, as the streaming kernel forms them), EXPAND back, and the
// Laplacian G0 - EXPAND(G1) of the tile weighted by w into the per-pixel sum
// A_w = sum over frames of lap0 * w.  The level-0 blend of the reference,
// acc0 = sum_k lap0_k * (w_k / N) (src/fuse/pyramid.zig:303-316, 1556-1603),
// equals A_w / N: N is the same for every frame at a pixel, so the division
// moves out of the sum (finalize0_kernel applies it once the weight sum is
// complete; the FP32 rounding of the two orders differs by a few ulp of the
// accumulator).  Where N stays <= 1e-12 the reference uses the mask 1/F for
// every frame instead; those pixels (in practice the window border of the
// ROI) also keep A_u = sum of lap0 in global memory, touched only while the
// weight sum so far is <= 1e-12 (it never decreases: the weights are
// non-negative).  Per frame the kernel keeps only w (for the mask pyramid of
// pass 2) and the level-1 Gaussian with its support (for the image pyramid
// of the levels above): no level-0 Laplacian, remapped frame or normalised
// mask goes through HBM.
namespace {

template <int B>
struct Lap0Layout {
  static constexpr int R0 = B > 4 ? B : 4;  // region halo left / top (REDUCE of the level-1 halo needs 4)
  static constexpr int R1 = B > 3 ? B : 3;  // right / bottom
  static constexpr int RW = TW + R0 + R1, RH = TH + R0 + R1;
  static constexpr int KS = kv_stride(RW);  // contrast-word row stride (odd words: distinct banks per row)
  static constexpr int CH = TH + 2 * B;     // rows of the window sums
  static constexpr int HS = TW + 1;
  static constexpr int NWIN = (2 * B + 1) * (2 * B + 1);
  static constexpr int RR = R0 - 4;         // region row / column of REDUCE tap 0 of halo output 0
  static constexpr int RRows = 2 * NH + 3;  // region rows the REDUCE reads
  static constexpr int TS = NW + 1;         // row stride of the horizontal REDUCE sums
};

template <int B>
struct __align__(16) Lap0Smem {
  using Lay = Lap0Layout<B>;
  uint32_t reg[Lay::RH * Lay::RW];   // remapped RGBA words of the region
  uint16_t kv[Lay::RH * Lay::KS];    // contrast words of the region
  union {
    struct {
      uint32_t h1[Lay::CH * Lay::HS];  // horizontal window sums: count | gray sum
      uint32_t h2[Lay::CH * Lay::HS];  // sum of gray^2
    } win;
    float hrow[NH * 3 * TW];           // horizontal EXPAND rows (after the window sums are used)
  } u;
  uint2 th[Lay::RRows * Lay::TS];    // horizontal REDUCE sums: R | G << 16, B | weight << 16
  float ng[3][NH * NW];              // level-1 Gaussian on the tile + 1-sample halo (0 outside the level)
  float inv_den[Lay::NWIN + 1];
};

template <typename T>
__device__ __forceinline__ void store_sample(void* plane, int64_t i, float v) { stv<T>((T*)plane, i, v); }

__device__ __forceinline__ void store_level_sample(void* plane, int storage, int64_t i, float v) {
  if (storage == FS_STORAGE_F16) store_sample<__half>(plane, i, v);
  else if (storage == FS_STORAGE_BF16) store_sample<__nv_bfloat16>(plane, i, v);
  else store_sample<float>(plane, i, v);
}

}  // namespace

template <int B, bool HARD>
__global__ void __launch_bounds__(NT, 2) lap0_kernel(const __grid_constant__ Lap0Args a) {
  using Lay = Lap0Layout<B>;
  constexpr int RW = Lay::RW, RH = Lay::RH, KS = Lay::KS, HS = Lay::HS, R0 = Lay::R0, TS = Lay::TS;
  extern __shared__ __align__(16) uint8_t smem_raw[];
  Lap0Smem<B>& S = *reinterpret_cast<Lap0Smem<B>*>(smem_raw);
  const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  const int x1 = x0 >> 1, y1 = y0 >> 1;
  for (int n = threadIdx.x; n <= Lay::NWIN; n += NT)
    S.inv_den[n] = n > 1 ? 1.0f / ((float)(n * (n - 1)) * 585225.0f) : 0.0f;
  // own pixels: column vc, rows vr0 .. vr0 + 7 of the tile (window sums,
  // weights, EXPAND and the blend all use this ownership)
  const int vc = threadIdx.x % TW, vr0 = (threadIdx.x / TW) * PPT;
  const int X = x0 + vc;
  float nacc[PPT], aw[PPT][3], wv[PPT];
  float best[HARD ? PPT : 1];      // hybrid: the winner's weight and RGBA word
  uint32_t hard[HARD ? PPT : 1];
  uint32_t umask = 0;
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    const int Y = y0 + vr0 + i;
    nacc[i] = 0.0f;
    aw[i][0] = aw[i][1] = aw[i][2] = 0.0f;
    if constexpr (HARD) {
      best[i] = -INFINITY;
      hard[i] = 0u;
    }
    if (!a.first && X < a.W && Y < a.H) {
      const int64_t o = (int64_t)Y * a.pitch + X;
      nacc[i] = a.norm[o];
      if (a.uni[o]) umask |= 1u << i;
#pragma unroll
      for (int c = 0; c < 3; ++c) aw[i][c] = a.aw[c * a.plane + o];
      if constexpr (HARD) {
        best[i] = a.best[o];
        hard[i] = a.hard[o];
      }
    }
  }
  __syncthreads();
  const bool exact = a.exact_expand != 0;
  for (int k = 0; k < a.K; ++k) {
    // A: the region's remapped words and contrast words
    load_region<RW, RH, KS, R0>(a.rgba[k], a.pitch, a.W, a.H, x0, y0, S.reg, S.kv);
    __syncthreads();
    // B: horizontal window sums (rows R0 - B .. R0 + TH + B - 1 of the
    // region, output columns c0 .. c0 + 7) and horizontal REDUCE sums (region
    // rows RR .. RR + 38, level-1 halo columns jj, jj + 1 from 7 taps)
    constexpr int kWinItems = Lay::CH * (TW / 8);
    constexpr int kRedItems = Lay::RRows * (NW / 2);
    for (int it = threadIdx.x; it < kWinItems + kRedItems; it += NT) {
      if (it < kWinItems) {
        const int r = it % Lay::CH, c0 = (it / Lay::CH) * 8;
        window_row8<B>(S.kv + (r + R0 - B) * KS + c0 + R0 - B, S.u.win.h1 + r * HS + c0, S.u.win.h2 + r * HS + c0);
      } else {
        const int j = it - kWinItems;
        const int r = j % Lay::RRows, jj = 2 * (j / Lay::RRows);
        const uint32_t* row = S.reg + (r + Lay::RR) * RW + 2 * jj + Lay::RR;
        uint32_t w7[7];
#pragma unroll
        for (int u = 0; u < 7; ++u) w7[u] = row[u];
        int4 hs[2];
        sum_row_u8(w7, 2, 1 << 30, hs);  // region words outside the ROI are 0 (no support)
#pragma unroll
        for (int h = 0; h < 2; ++h)
          S.th[r * TS + jj + h] = make_uint2((uint32_t)hs[h].x | ((uint32_t)hs[h].y << 16),
                                             (uint32_t)hs[h].z | ((uint32_t)hs[h].w << 16));
      }
    }
    __syncthreads();
    // C1: vertical window sums -> this frame's weights of the own pixels
    {
      uint32_t p = 0, q = 0;
#pragma unroll
      for (int t = 0; t <= 2 * B; ++t) {
        p += S.u.win.h1[(vr0 + t) * HS + vc];
        q += S.u.win.h2[(vr0 + t) * HS + vc];
      }
      float* wout = a.w[k];
#pragma unroll
      for (int i = 0; i < PPT; ++i) {
        if (i > 0) {
          p += S.u.win.h1[(vr0 + i + 2 * B) * HS + vc] - S.u.win.h1[(vr0 + i - 1) * HS + vc];
          q += S.u.win.h2[(vr0 + i + 2 * B) * HS + vc] - S.u.win.h2[(vr0 + i - 1) * HS + vc];
        }
        const int Y = y0 + vr0 + i;
        wv[i] = 0.0f;
        if (X >= a.W || Y >= a.H) continue;
        const uint32_t own = S.reg[(vr0 + i + R0) * RW + (vc + R0)];
        const uint32_t al = px_alpha(own);
        float w = 0.0f;
        if (a.window_ok && al > 0 && X >= B && Y >= B && X < a.W - B && Y < a.H - B)
          w = __fmul_rn(window_stddev<B>(p, q, S.inv_den), alpha_support(al));
        wv[i] = w;
        if constexpr (HARD) {
          if (w > best[i]) {  // strictly larger weights win (src/fuse/blend.zig:259-261)
            best[i] = w;
            hard[i] = own;
          }
        }
        nacc[i] = __fadd_rn(nacc[i], w);
        if (al > 0) umask |= 1u << i;
        wout[(int64_t)Y * a.pitch + X] = w;
      }
    }
    // C2: vertical REDUCE -> level-1 Gaussian of the tile and its halo
    // (rows ii, ii + 1 per item), the tile's own samples stored for the
    // levels above
    {
      const LevelPlanes& g1 = a.g1[k];
      for (int it = threadIdx.x; it < (NH / 2) * NW; it += NT) {
        const int ii = 2 * (it / NW), jj = it % NW;
        uint2 t[7];
#pragma unroll
        for (int u = 0; u < 7; ++u) t[u] = S.th[(2 * ii + u) * TS + jj];
        const int xj = x1 - 1 + jj;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          uint32_t sx = 0, sy = 0;
#pragma unroll
          for (int ky = 0; ky < 5; ++ky) {
            sx += (uint32_t)kwi(ky) * t[2 * h + ky].x;  // 16-bit lanes stay below 2^16
            sy += (uint32_t)kwi(ky) * t[2 * h + ky].y;
          }
          const int yi = y1 - 1 + ii + h;
          const float ws = small_int_float((int)(sy >> 16));
          const bool sup = xj >= 0 && yi >= 0 && xj < a.wn && yi < a.hn && ws > 0.f;
          const float rc = sup ? __fdividef(1.0f, ws) : 0.0f;
          const float g[3] = {small_int_float((int)(sx & 0xFFFFu)) * rc, small_int_float((int)(sx >> 16)) * rc,
                              small_int_float((int)(sy & 0xFFFFu)) * rc};
          const int o = (ii + h) * NW + jj;
#pragma unroll
          for (int c = 0; c < 3; ++c) S.ng[c][o] = g[c];
          if (ii + h >= 1 && ii + h <= TH1 && jj >= 1 && jj <= TW1 && xj < a.wn && yi < a.hn) {
            const int64_t go = (int64_t)yi * a.pitch_n + xj;
#pragma unroll
            for (int c = 0; c < 3; ++c) store_level_sample(g1.g, a.storage, c * g1.plane + go, g[c]);
            g1.s[go] = sup ? 1 : 0;
          }
        }
      }
    }
    __syncthreads();
    // D: horizontal EXPAND of the level-1 rows (the operations of
    // expand_blend_step)
    float* hrow = S.u.hrow;
    for (int i = threadIdx.x; i < NH * (TW / 2); i += NT) {
      const int ii = i / (TW / 2), pp = i % (TW / 2);
      const int yi = y1 - 1 + ii;
      if (yi < 0 || yi >= a.hn) continue;
      const int j = x1 + pp, o = x1 - 1;
      int ia, ib, ic;
      if (exact) {
        ia = pp;
        ib = pp + 1;
        ic = pp + 2;
      } else {
        ia = clampi(j - 1, 0, a.wn - 1) - o;
        ib = clampi(j, 0, a.wn - 1) - o;
        ic = clampi(j + 1, 0, a.wn - 1) - o;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float* g = S.ng[c] + ii * NW;
        const float A = g[ia], Bv = g[ib], C = g[ic];
        float ev, od;
        if (exact) {
          ev = __fadd_rn(__fadd_rn(A, __fmul_rn(6.0f, Bv)), C);
          od = __fmul_rn(4.0f, __fadd_rn(Bv, C));
        } else {
          ev = __fmul_rn(__fadd_rn(__fadd_rn(A, __fmul_rn(6.0f, Bv)), C), 0.125f);
          od = __fmul_rn(__fadd_rn(Bv, C), 0.5f);
        }
        hrow[(ii * 3 + c) * TW + 2 * pp] = ev;
        hrow[(ii * 3 + c) * TW + 2 * pp + 1] = od;
      }
    }
    __syncthreads();
    // E: vertical EXPAND down the own strip, Laplacian, A_w += lap0 * w
    {
      const int q0 = (y0 + vr0) >> 1;
      constexpr int NR = PPT / 2 + 2;
      float hv[3][NR];
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        int q = q0 - 1 + r;
        bool zero = false;
        if (exact) zero = q < 0 || q >= a.hn;
        else q = clampi(q, 0, a.hn - 1);
        const int lr = q - (y1 - 1);
#pragma unroll
        for (int c = 0; c < 3; ++c) hv[c][r] = zero ? 0.0f : hrow[(lr * 3 + c) * TW + vc];
      }
      const bool first_frame = a.first && k == 0;
#pragma unroll
      for (int i = 0; i < PPT; ++i) {
        const int y = y0 + vr0 + i;
        if (X >= a.W || y >= a.H) continue;
        const int j = i >> 1;
        const float div = exact ? exact_expand_divisor(X, y, a.wn, a.hn) : 1.0f;
        const uint32_t g0 = S.reg[(vr0 + i + R0) * RW + (vc + R0)];
        const bool fallback = nacc[i] <= 1e-12f;  // the weight sum so far: A_u still needed here
        const int64_t o = (int64_t)y * a.pitch + X;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float e;
          if ((i & 1) == 0) {
            const float v = __fadd_rn(__fadd_rn(hv[c][j], __fmul_rn(6.0f, hv[c][j + 1])), hv[c][j + 2]);
            e = exact ? __fdiv_rn(v, div) : __fmul_rn(v, 0.125f);
          } else if (exact) {
            e = __fdiv_rn(__fadd_rn(hv[c][j + 1], hv[c][j + 2]), div);
          } else {
            e = __fmul_rn(__fadd_rn(hv[c][j + 1], hv[c][j + 1]), 0.5f);
          }
          const float lap = __fsub_rn(chf(g0, c), e);
          aw[i][c] = __fadd_rn(aw[i][c], __fmul_rn(lap, wv[i]));
          if (fallback) {
            float* pu = a.au + c * a.plane + o;
            *pu = first_frame ? lap : __fadd_rn(*pu, lap);
          }
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    const int Y = y0 + vr0 + i;
    if (X < a.W && Y < a.H) {
      const int64_t o = (int64_t)Y * a.pitch + X;
      a.norm[o] = nacc[i];
      a.uni[o] = (uint8_t)((umask >> i) & 1u);
#pragma unroll
      for (int c = 0; c < 3; ++c) a.aw[c * a.plane + o] = aw[i][c];
      if constexpr (HARD) {
        a.best[o] = best[i];
        a.hard[o] = hard[i];
      }
    }
  }
}

template <int B, bool HARD>
static cudaError_t launch_lap0_bh(const Lap0Args& a, cudaStream_t s) {
  static DeviceOnce configured;
  const size_t sm = sizeof(Lap0Smem<B>);
  cudaError_t e = configure(lap0_kernel<B, HARD>, sm, &configured);
  if (e != cudaSuccess) return e;
  dim3 grid((a.W + TW - 1) / TW, (a.H + TH - 1) / TH);
  lap0_kernel<B, HARD><<<grid, NT, sm, s>>>(a);
  return cudaGetLastError();
}
template <int B>
static cudaError_t launch_lap0_b(const Lap0Args& a, cudaStream_t s) {
  return a.best ? launch_lap0_bh<B, true>(a, s) : launch_lap0_bh<B, false>(a, s);
}

cudaError_t launch_lap0(const Lap0Args& a, int border, cudaStream_t s) {
  if (a.K < 1 || a.K > kMaxBatch) return cudaErrorInvalidValue;
  switch (border) {
    case 1: return launch_lap0_b<1>(a, s);
    case 2: return launch_lap0_b<2>(a, s);
    case 3: return launch_lap0_b<3>(a, s);
    case 4: return launch_lap0_b<4>(a, s);
    case 5: return launch_lap0_b<5>(a, s);
    case 6: return launch_lap0_b<6>(a, s);
    case 7: return launch_lap0_b<7>(a, s);
    default: return cudaErrorInvalidValue;
  }
}

// Level-0 accumulator of a LAPS stack once the weight sum N is complete:
// acc0 = A_w / N where N > 1e-12, else A_u / F (the reference's mask 1/F for
// every frame), written over A_w (acc0 and A_w share the buffer).
__global__ void finalize0_kernel(float* acc, const float* au, const float* norm, int64_t plane, int64_t pitch, int w,
                                 int h, float inv_count) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)w * h) return;
  const int64_t o = (i / w) * pitch + i % w;
  const float nv = norm[o];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t q = c * plane + o;
    acc[q] = nv > 1e-12f ? __fdiv_rn(acc[q], nv) : __fmul_rn(au[q], inv_count);
  }
}

cudaError_t launch_finalize0(float* acc, const float* au, const float* norm, int64_t plane, int64_t pitch, int w,
                             int h, float inv_count, cudaStream_t s) {
  const int64_t n = (int64_t)w * h;
  finalize0_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(acc, au, norm, plane, pitch, w, h, inv_count);
  return cudaGetLastError();
}

// ================================================================ collapse
// parent += EXPAND(child) in place (src/fuse/pyramid.zig:223-248); at level
// 0 also quantise trunc(clamp(v + 0.5, 0, 255)) into interleaved RGB.
__global__ void __launch_bounds__(NT) collapse_kernel(const __grid_constant__ CollapseArgs a) {
  __shared__ float cg[3][NH * NW];
  __shared__ float hrow[NH * 3 * TW];
  const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  const int x1 = x0 >> 1, y1 = y0 >> 1;
  const bool exact = a.exact_expand != 0;
  for (int i = threadIdx.x; i < NH * NW; i += NT) {
    const int X = x1 - 1 + i % NW, Y = y1 - 1 + i / NW;
    const bool in = X >= 0 && Y >= 0 && X < a.wc && Y < a.hc;
    const int64_t o = (int64_t)Y * a.pitch_c + X;
    for (int c = 0; c < 3; ++c) cg[c][i] = in ? a.acc_c[c * a.plane_c + o] : 0.0f;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NH * TW; i += NT) {
    const int ii = i / TW, xx = i % TW;
    const int yi = y1 - 1 + ii;
    if (yi < 0 || yi >= a.hc) continue;
    const Taps t = expand_taps(x0 + xx, x1, a.wc, exact);
    for (int c = 0; c < 3; ++c) hrow[(ii * 3 + c) * TW + xx] = expand_h1(cg[c] + ii * NW, t, exact);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < TH * TW; i += NT) {
    const int yy = i / TW, xx = i % TW;
    const int x = x0 + xx, y = y0 + yy;
    if (x >= a.wp || y >= a.hp) continue;
    const int64_t o = (int64_t)y * a.pitch_p + x;
    const Rows r = expand_rows(y, y1, a.hc, exact);
    const float div = exact ? exact_expand_divisor(x, y, a.wc, a.hc) : 1.0f;
    for (int c = 0; c < 3; ++c) {
      const float v = expand_v1(hrow + c * TW + xx, 3 * TW, r, exact, div);
      float* p = a.acc_p + c * a.plane_p + o;
      const float nv = __fadd_rn(*p, v);
      if (a.out) {
        if (a.out16) {
          const float q = fminf(fmaxf(__fadd_rn(nv, 0.5f), 0.0f), 65535.0f);
          reinterpret_cast<uint16_t*>(a.out + (int64_t)y * a.out_pitch)[(int64_t)x * 3 + c] = (uint16_t)q;
        } else {
          const float q8 = fminf(fmaxf(__fadd_rn(nv, 0.5f), 0.0f), 255.0f);
          a.out[(int64_t)y * a.out_pitch + (int64_t)x * 3 + c] = (uint8_t)q8;
        }
        if (a.base) a.base[(int64_t)y * a.base_pitch + (int64_t)x * 3 + c] = nv;
      } else {
        *p = nv;
      }
    }
  }
}

// The clamped-EXPAND collapse step (parent side > 512), streaming: each
// thread owns parent columns 2j, 2j + 1 (child columns j - 1 .. j + 1,
// clamped) and walks a strip of parent rows, keeping the horizontal EXPAND of
// child rows q - 1, q, q + 1 in registers; parent row 2q takes all three,
// row 2q + 1 row q twice.  Every operation is collapse_kernel's clamped one
// (expand_h1, expand_v1), in its order.
constexpr int kCollapseRows = 32;  // parent rows per strip (even)

__device__ __forceinline__ void collapse_hrow(const CollapseArgs& a, int q, int jl, int jc, int jr,
                                              float (&h)[3][2]) {
  const int r = clampi(q, 0, a.hc - 1);
  const float* row = a.acc_c + (int64_t)r * a.pitch_c;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float* g = row + c * a.plane_c;
    const float g0 = g[jl], g1 = g[jc], g2 = g[jr];
    h[c][0] = __fmul_rn(__fadd_rn(__fadd_rn(g0, __fmul_rn(6.0f, g1)), g2), 0.125f);
    h[c][1] = __fmul_rn(__fadd_rn(g1, g2), 0.5f);
  }
}

__global__ void __launch_bounds__(128) collapse_stream_kernel(const __grid_constant__ CollapseArgs a) {
  const int j = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int x = 2 * j;
  if (x >= a.wp) return;  // no barriers below
  const bool two = x + 1 < a.wp;
  const int jl = max(j - 1, 0), jc = min(j, a.wc - 1), jr = min(j + 1, a.wc - 1);
  const int y0 = (int)blockIdx.y * kCollapseRows;
  const int y1 = min(y0 + kCollapseRows, a.hp);
  float hm[3][2], hc[3][2], hn[3][2];
  int q = y0 >> 1;
  collapse_hrow(a, q - 1, jl, jc, jr, hm);
  collapse_hrow(a, q, jl, jc, jr, hc);
  collapse_hrow(a, q + 1, jl, jc, jr, hn);
  for (int y = y0; y < y1; y += 2, ++q) {
#pragma unroll
    for (int yy = 0; yy < 2; ++yy) {
      const int yr = y + yy;
      if (yr >= y1) break;
      float v[3][2];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int u = 0; u < 2; ++u)
          v[c][u] = yy == 0 ? __fmul_rn(__fadd_rn(__fadd_rn(hm[c][u], __fmul_rn(6.0f, hc[c][u])), hn[c][u]), 0.125f)
                            : hc[c][u];  // the reference's (H + H) * 0.5, which is H exactly
      const int64_t o = (int64_t)yr * a.pitch_p + x;
      float nv[3][2];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float* p = a.acc_p + c * a.plane_p + o;
        if (two) {
          const float2 pv = *reinterpret_cast<const float2*>(p);  // x even, pitch a multiple of 32
          nv[c][0] = __fadd_rn(pv.x, v[c][0]);
          nv[c][1] = __fadd_rn(pv.y, v[c][1]);
          if (!a.out) *reinterpret_cast<float2*>(p) = make_float2(nv[c][0], nv[c][1]);
        } else {
          nv[c][0] = __fadd_rn(p[0], v[c][0]);
          nv[c][1] = 0.0f;
          if (!a.out) p[0] = nv[c][0];
        }
      }
      if (a.out) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          if (u == 1 && !two) break;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int64_t ob = (int64_t)(x + u) * 3 + c;
            if (a.out16) {
              const float q16 = fminf(fmaxf(__fadd_rn(nv[c][u], 0.5f), 0.0f), 65535.0f);
              reinterpret_cast<uint16_t*>(a.out + (int64_t)yr * a.out_pitch)[ob] = (uint16_t)q16;
            } else {
              const float q8 = fminf(fmaxf(__fadd_rn(nv[c][u], 0.5f), 0.0f), 255.0f);
              a.out[(int64_t)yr * a.out_pitch + ob] = (uint8_t)q8;
            }
            if (a.base) a.base[(int64_t)yr * a.base_pitch + ob] = nv[c][u];
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        hm[c][u] = hc[c][u];
        hc[c][u] = hn[c][u];
      }
    if (y + 2 < y1) collapse_hrow(a, q + 2, jl, jc, jr, hn);
  }
}

cudaError_t launch_collapse(const CollapseArgs& a, cudaStream_t s) {
  if (!a.exact_expand) {
    const dim3 grid((unsigned)((a.wp + 255) / 256), (unsigned)((a.hp + kCollapseRows - 1) / kCollapseRows));
    collapse_stream_kernel<<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
  }
  dim3 grid((a.wp + TW - 1) / TW, (a.hp + TH - 1) / TH);
  collapse_kernel<<<grid, NT, 0, s>>>(a);
  return cudaGetLastError();
}

// Quantise a single-level accumulator (1x1 images have no collapse step).
__global__ void quantize_kernel(const float* acc, int64_t plane, int64_t pitch, int w, int h, uint8_t* out,
                                int64_t out_pitch, float* base, int64_t base_pitch, int out16) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w * h) return;
  const int x = i % w, y = i / w;
  for (int c = 0; c < 3; ++c) {
    const float v = acc[c * plane + (int64_t)y * pitch + x];
    if (out16)
      reinterpret_cast<uint16_t*>(out + (int64_t)y * out_pitch)[x * 3 + c] =
          (uint16_t)fminf(fmaxf(__fadd_rn(v, 0.5f), 0.0f), 65535.0f);
    else
      out[(int64_t)y * out_pitch + x * 3 + c] = (uint8_t)fminf(fmaxf(__fadd_rn(v, 0.5f), 0.0f), 255.0f);
    if (base) base[(int64_t)y * base_pitch + x * 3 + c] = v;
  }
}

cudaError_t launch_quantize(const float* acc, int64_t plane, int64_t pitch, int w, int h, uint8_t* out,
                            int64_t out_pitch, float* base, int64_t base_pitch, int out16, cudaStream_t s) {
  quantize_kernel<<<(w * h + 255) / 256, 256, 0, s>>>(acc, plane, pitch, w, h, out, out_pitch, base, base_pitch,
                                                      out16);
  return cudaGetLastError();
}

// ================================================================ hybrid
// hybrid-pyramid-contrast (src/stack/pipeline.zig:177-236): the
// pyramid-contrast image ("soft"), the hardmask-contrast image ("hard": per
// pixel the colour of the first frame, in order, with the strictly largest
// weight x alpha support, blend.updateWinners, src/fuse/blend.zig:188-289)
// and their Laplacian merge (mergeHybridImages, src/fuse/pyramid.zig:271-301).

// Winners over a batch's pass-2 planes (remapped RGBA word and alpha-weighted
// contrast: the reference's effectiveWeightU8 of the same weight).
struct WinnersArgs {
  FramePlanes planes[kMaxBatch];
  int32_t K, first, w, h;
  int64_t pitch;
  float* best;
  uint32_t* hard;
};

__global__ void winners_kernel(const __grid_constant__ WinnersArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)a.w * a.h) return;
  const int64_t o = (i / a.w) * a.pitch + i % a.w;
  float b = a.first ? -INFINITY : a.best[o];
  uint32_t hw = a.first ? 0u : a.hard[o];
  for (int k = 0; k < a.K; ++k) {
    const float wk = a.planes[k].w[o];
    if (wk > b) {
      b = wk;
      hw = a.planes[k].rgba[o];
    }
  }
  a.best[o] = b;
  a.hard[o] = hw;
}

cudaError_t launch_winners(const FramePlanes* planes, int K, float* best, uint32_t* hard, int first, int w, int h,
                           int64_t pitch, cudaStream_t s) {
  if (K < 1 || K > kMaxBatch) return cudaErrorInvalidValue;
  WinnersArgs a;
  for (int k = 0; k < K; ++k) a.planes[k] = planes[k];
  a.K = K;
  a.first = first;
  a.w = w;
  a.h = h;
  a.pitch = pitch;
  a.best = best;
  a.hard = hard;
  const int64_t n = (int64_t)w * h;
  winners_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}

__global__ void rgb_to_planes_kernel(const uint8_t* src, int64_t src_pitch, int px_bytes, float* dst, int64_t plane,
                                     int64_t pitch, int w, int h) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)w * h) return;
  const int64_t x = i % w, y = i / w;
  const uint8_t* p = src + y * src_pitch + x * px_bytes;
  const int64_t o = y * pitch + x;
#pragma unroll
  for (int c = 0; c < 3; ++c) dst[c * plane + o] = (float)p[c];
}

cudaError_t launch_rgb_to_planes(const uint8_t* src, int64_t src_pitch, int px_bytes, float* dst, int64_t plane,
                                 int64_t pitch, int w, int h, cudaStream_t s) {
  const int64_t n = (int64_t)w * h;
  rgb_to_planes_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, src_pitch, px_bytes, dst, plane, pitch, w,
                                                                   h);
  return cudaGetLastError();
}

namespace {
__device__ __forceinline__ int clamp_coord(int c, int limit) { return c <= 0 ? 0 : (c >= limit ? limit - 1 : c); }
// (a + 4 b + 6 c + 4 d + e) * (1 / 16), left to right, no contraction
__device__ __forceinline__ float five_tap(float a, float b, float c, float d, float e) {
  float v = __fadd_rn(a, __fmul_rn(4.0f, b));
  v = __fadd_rn(v, __fmul_rn(6.0f, c));
  v = __fadd_rn(v, __fmul_rn(4.0f, d));
  v = __fadd_rn(v, e);
  return __fmul_rn(v, 0.0625f);
}
}  // namespace

// One output sample per thread: five clamped source rows, each reduced
// horizontally (horizontalReduceRgbRow), then combined vertically.
__global__ void reduce_plain_kernel(const float* src, int64_t splane, int64_t spitch, int sw, int sh, float* dst,
                                    int64_t dplane, int64_t dpitch, int dw, int dh) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)dw * dh) return;
  const int dx = (int)(i % dw), dy = (int)(i / dw);
  int xs[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) xs[k] = clamp_coord(2 * dx + k - 2, sw);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float* pl = src + c * splane;
    float r[5];
#pragma unroll
    for (int ky = 0; ky < 5; ++ky) {
      const float* row = pl + (int64_t)clamp_coord(2 * dy + ky - 2, sh) * spitch;
      r[ky] = five_tap(row[xs[0]], row[xs[1]], row[xs[2]], row[xs[3]], row[xs[4]]);
    }
    dst[c * dplane + (int64_t)dy * dpitch + dx] = five_tap(r[0], r[1], r[2], r[3], r[4]);
  }
}

cudaError_t launch_reduce_plain(const float* src, int64_t splane, int64_t spitch, int sw, int sh, float* dst,
                                int64_t dplane, int64_t dpitch, int dw, int dh, cudaStream_t s) {
  const int64_t n = (int64_t)dw * dh;
  reduce_plain_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, splane, spitch, sw, sh, dst, dplane, dpitch,
                                                                  dw, dh);
  return cudaGetLastError();
}

// Laplacians of the soft and hard pyramids at level l (G_l - EXPAND(G_{l+1}),
// expandRgb in both boundary modes, the operations of collapse_kernel) and
// the merged level: soft + (hard - soft) * mix inside the hard range, soft
// elsewhere.
__global__ void __launch_bounds__(NT) merge_level_kernel(const __grid_constant__ MergeArgs a) {
  __shared__ float cg[2][3][NH * NW];
  __shared__ float hrow[2][NH * 3 * TW];
  const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  const int x1 = x0 >> 1, y1 = y0 >> 1;
  const bool exact = a.exact_expand != 0;
  for (int i = threadIdx.x; i < NH * NW; i += NT) {
    const int X = x1 - 1 + i % NW, Y = y1 - 1 + i / NW;
    const bool in = X >= 0 && Y >= 0 && X < a.wc && Y < a.hc;
    const int64_t o = (int64_t)Y * a.pitch_c + X;
    for (int c = 0; c < 3; ++c) {
      cg[0][c][i] = in ? a.soft_c[c * a.plane_c + o] : 0.0f;
      cg[1][c][i] = in ? a.hard_c[c * a.plane_c + o] : 0.0f;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NH * TW; i += NT) {
    const int ii = i / TW, xx = i % TW;
    const int yi = y1 - 1 + ii;
    if (yi < 0 || yi >= a.hc) continue;
    const Taps t = expand_taps(x0 + xx, x1, a.wc, exact);
    for (int v = 0; v < 2; ++v)
      for (int c = 0; c < 3; ++c) hrow[v][(ii * 3 + c) * TW + xx] = expand_h1(cg[v][c] + ii * NW, t, exact);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < TH * TW; i += NT) {
    const int yy = i / TW, xx = i % TW;
    const int x = x0 + xx, y = y0 + yy;
    if (x >= a.wp || y >= a.hp) continue;
    const int64_t o = (int64_t)y * a.pitch_p + x;
    const Rows r = expand_rows(y, y1, a.hc, exact);
    const float div = exact ? exact_expand_divisor(x, y, a.wc, a.hc) : 1.0f;
    for (int c = 0; c < 3; ++c) {
      const float ls = __fsub_rn(a.soft_p[c * a.plane_p + o], expand_v1(hrow[0] + c * TW + xx, 3 * TW, r, exact, div));
      const float lh = __fsub_rn(a.hard_p[c * a.plane_p + o], expand_v1(hrow[1] + c * TW + xx, 3 * TW, r, exact, div));
      a.acc[c * a.plane_p + o] = a.mixed ? __fadd_rn(ls, __fmul_rn(__fsub_rn(lh, ls), a.mix)) : ls;
    }
  }
}

cudaError_t launch_merge_level(const MergeArgs& a, cudaStream_t s) {
  dim3 grid((a.wp + TW - 1) / TW, (a.hp + TH - 1) / TH);
  merge_level_kernel<<<grid, NT, 0, s>>>(a);
  return cudaGetLastError();
}

__global__ void merge_top_kernel(const float* soft, const float* hard, float* acc, int64_t plane, int64_t pitch, int w,
                                 int h, int mixed, float mix) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)w * h) return;
  const int64_t o = (i / w) * pitch + i % w;
  for (int c = 0; c < 3; ++c) {
    const float sv = soft[c * plane + o], hv = hard[c * plane + o];
    acc[c * plane + o] = mixed ? __fadd_rn(sv, __fmul_rn(__fsub_rn(hv, sv), mix)) : sv;
  }
}

cudaError_t launch_merge_top(const float* soft, const float* hard, float* acc, int64_t plane, int64_t pitch, int w,
                             int h, int mixed, float mix, cudaStream_t s) {
  const int64_t n = (int64_t)w * h;
  merge_top_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(soft, hard, acc, plane, pitch, w, h, mixed, mix);
  return cudaGetLastError();
}

// ========================================================== mask support
// Support of the mask pyramid (frame independent): a level-(l+1) sample is
// supported when any in-range 5x5 tap below it is (src/fuse/pyramid.zig:1032-1040).
__global__ void mask_support_kernel(const __grid_constant__ MaskSupportArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.dw * a.dh) return;
  const int x = i % a.dw, y = i / a.dw;
  uint8_t any = 0;
  for (int ky = 0; ky < 5 && !any; ++ky) {
    const int sy = 2 * y - 2 + ky;
    if (sy < 0 || sy >= a.sh) continue;
    for (int kx = 0; kx < 5; ++kx) {
      const int sx = 2 * x - 2 + kx;
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
  const int n = a.dw * a.dh;
  mask_support_kernel<<<(n + 255) / 256, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// ============================================================ remap only
// Standalone remap (src/remap.zig:166-278): ROI-sized output with
// channels + 1 samples per pixel.
__global__ void __launch_bounds__(NT) remap_kernel(const __grid_constant__ RemapArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = NT / 32;
  const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  constexpr int NBX = TW / 8, NBY = TH / 4, NB = NBX * NBY;
  const bool fast_ok = a.f.warp.kind == WARP_HOMOGRAPHY && !a.f.warp.guard;
  const int du = lane & 7, dv = lane >> 3;
  __shared__ Anchor anchor[NB];
  for (int b = threadIdx.x; b < NB; b += NT) {
    bool ok = false;
    Anchor an = {};
    if (fast_ok) an = make_anchor(a.f.warp, x0 + (b % NBX) * 8, y0 + (b / NBX) * 4, &ok);
    if (!ok) an.ix = kNoAnchor;
    anchor[b] = an;
  }
  __syncthreads();
  for (int blk = warp; blk < NB; blk += nwarps) {
    const int X = x0 + (blk % NBX) * 8 + du, Y = y0 + (blk / NBX) * 4 + dv;
    if (X >= a.W || Y >= a.H) continue;
    const Anchor an = anchor[blk];
    const uint32_t v = an.ix != kNoAnchor ? sample_fast(a.f.warp, a.f.src, an, du, dv, X, Y)
                                          : sample_exact(a.f.warp, a.f.src, X, Y);
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

cudaError_t launch_remap(const RemapArgs& a, cudaStream_t s) {
  dim3 grid((a.W + TW - 1) / TW, (a.H + TH - 1) / TH);
  remap_kernel<<<grid, NT, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace fs
