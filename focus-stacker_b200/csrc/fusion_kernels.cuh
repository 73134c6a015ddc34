// Kernel argument records and launchers of the fusion path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/focuscuda.h"
#include "fs_common.h"
#include "remap_device.cuh"

namespace fs {

static constexpr int kMaxBatch = 8;   // frames per pass over per-pixel state (K)
static constexpr int kTileW = 64;     // output tile of every 2-D kernel
static constexpr int kTileH = 32;
static constexpr int kThreads = 256;
static constexpr int kMaxBorder = 7;  // contrast windows 3 .. 15

// One input frame of a batch.
struct FrameIn {
  SrcImage src;   // source frame (remap) or aligned frame (RGBA / RGB)
  Warp warp;      // kind WARP_ALIGNED for aligned input
};

// Pass-1 product of one frame kept for pass 2: the remapped frame as packed
// RGBA words (R | G << 8 | B << 16 | A << 24) and its alpha-weighted local
// contrast, on the level-0 grid.
struct FramePlanes {
  uint32_t* rgba;
  float* w;
};

// Planes of one pyramid level l >= 1 of one frame: RGB Gaussian (3 planes),
// normalised mask, image support.  g / m hold `storage` elements.
struct LevelPlanes {
  void* g;
  void* m;
  uint8_t* s;
  int64_t plane;  // elements per colour plane (h * pitch)
};

struct RemapWeightArgs {
  int32_t W, H;          // ROI (level 0) size
  int32_t window_ok;     // W >= window && H >= window
  int32_t K;             // frames in this batch
  int32_t accumulate;    // 1: add weights into the weight sum / union (pass 1)
  int32_t first;         // 1: the sums start at zero
  float* norm;
  uint8_t* uni;
  int64_t pitch;         // level-0 row pitch (elements; bytes for u8 planes)
  FrameIn f[kMaxBatch];
  FramePlanes out[kMaxBatch];  // null members: do not store
  // the batch's exact-sample queue (remap_tile_kernel hands the samples its
  // fast path cannot decide to remap_exact_kernel): frame << 48 | Y << 24 |
  // X per entry, exact_n entries reserved of exact_cap; null: each CTA takes
  // its own undecided samples exactly
  uint64_t* exact_q;
  uint32_t* exact_n;
  uint32_t exact_cap;
};
// Entries of the exact-sample queue per 64x32 tile and frame of a batch
// (about 3 are used under the synthetic stacks' warps; a CTA whose samples
// do not fit takes them itself).
static constexpr uint32_t kExactPerTile = 16;

struct LevelArgs {
  int32_t level;         // l: this launch reads level l, writes level l + 1
  int32_t levels;        // L
  int32_t wl, hl;        // level l size
  int32_t wn, hn;        // level l + 1 size
  int64_t pitch_l, pitch_n;   // elements per row; u8 planes use the same pitch in bytes
  int32_t exact_expand;  // max(wl, hl) <= 512: no-wrap expand back to level l
  int32_t K;
  // level 0
  float inv_count;       // 1 / N (f32), the reference's default weight
  const float* norm;
  FramePlanes in0[kMaxBatch];
  // level >= 1 inputs (per frame in batch)
  LevelPlanes in[kMaxBatch];
  // outputs at level l + 1 (per frame in batch)
  LevelPlanes out[kMaxBatch];
  const uint8_t* sm_l;   // mask support at level l (union at level 0)
  float* acc_l;          // accumulator level l, 3 planes
  int64_t acc_plane_l;
  float* acc_n;          // accumulator level l + 1 (used when l + 1 is the top level)
  int64_t acc_plane_n;
  // frame-parallel launch (grid.z = K, one frame per CTA): each frame's
  // blend contribution goes to contrib[k] (3 planes of acc_plane_l floats;
  // contrib_top[k], 3 planes of acc_plane_n, for the top level) and
  // launch_sum_contrib adds them to the accumulator in frame order
  int32_t frame_parallel;
  float* contrib;
  float* contrib_top;
  // split pyramid (launch_img_level): frame k's Laplacian planes at level l
  // (3 planes of acc_plane_l samples in the level storage type) and its top
  // Gaussian (3 planes of acc_plane_n floats, written when l + 1 is the top)
  void* lap[kMaxBatch];
  float* gtop[kMaxBatch];
};

// Fused pass 1 of the LAPS mode (lap0_kernel): a batch of frames remapped,
// weighted, reduced to level 1 and blended at level 0 as A_w += lap0 * w.
struct Lap0Args {
  int32_t W, H;            // ROI (level 0) size
  int32_t window_ok;       // W >= window && H >= window
  int32_t K;               // frames in this batch
  int32_t first;           // 1: first batch of the stack (sums start at zero)
  int32_t exact_expand;    // max(W, H) <= 512: no-wrap EXPAND back to level 0
  int32_t wn, hn;          // level-1 size
  int32_t storage;         // level-1 Gaussian storage (fs_level_storage)
  int32_t pad0;
  int64_t pitch, pitch_n;  // level-0 / level-1 row pitch (elements)
  int64_t plane;           // level-0 plane (pitch * H elements)
  float* norm;             // weight sum N
  uint8_t* uni;            // union support
  float* aw;               // A_w = sum of lap0 * w, 3 planes
  float* au;               // A_u = sum of lap0 while N <= 1e-12, 3 planes
  const uint32_t* rgba[kMaxBatch];  // per frame: its remapped RGBA plane (remap_tile_kernel)
  float* w[kMaxBatch];         // per frame: its level-0 weight plane
  LevelPlanes g1[kMaxBatch];   // per frame: level-1 Gaussian (storage) and support
  // hybrid method only (null otherwise): per pixel the largest weight so far
  // and the RGBA word of the frame that holds it (blend.updateWinners)
  float* best;
  uint32_t* hard;
};

struct CollapseArgs {
  int32_t wp, hp, wc, hc;     // parent / child sizes
  int64_t pitch_p, pitch_c;
  int32_t exact_expand;       // max(wp, hp) <= 512
  float* acc_p;               // parent accumulator (updated in place)
  int64_t plane_p;
  const float* acc_c;
  int64_t plane_c;
  uint8_t* out;               // final level: interleaved RGB output (u8, or u16 with out16), else null
  int64_t out_pitch;          // bytes per output row
  int32_t out16;              // 1: u16 output samples (clamped to 65535), 0: u8
  float* base;                // final level, optional: collapsed base before quantisation (RGB f32)
  int64_t base_pitch;         // elements per row
};

// Mask REDUCE of one level for every frame of a stack, one frame per grid z:
// level-(l+1) mask = support-weighted 5x5 REDUCE of the level-l mask with the
// level-l union support (src/fuse/pyramid.zig:997-1043), the products and
// sums of the level kernels' mask REDUCE in the same order.
struct MaskReduceArgs {
  const void* const* in;  // per frame: level-l mask (l >= 1)
  void* const* out;       // per frame: level-(l+1) mask
  const uint8_t* sm;      // level-l union support
  int32_t wl, hl, wn, hn;
  int64_t pitch_l, pitch_n;
};
// Storage of in / out masks: 0 f32, 1 f16, 2 bf16.
cudaError_t launch_mask_reduce(const MaskReduceArgs& a, int frames, int in_storage, int out_storage, cudaStream_t s);

struct MaskSupportArgs {
  const uint8_t* src;
  int32_t sw, sh;
  int64_t spitch;
  uint8_t* dst;
  int32_t dw, dh;
  int64_t dpitch;
};

struct RemapArgs {
  FrameIn f;
  int32_t W, H;       // output size
  uint8_t* dst;
  int64_t dst_pitch;
  int32_t dst_ch;     // channels + 1
};

cudaError_t launch_remap_weights(const RemapWeightArgs& a, int border, cudaStream_t s);
// The remap alone (the RGBA planes; norm, uni and the weight planes untouched).
cudaError_t launch_remap_tiles(const RemapWeightArgs& a, cudaStream_t s);

// 16-bit frames (fusion16.cu): pass 1 (accumulate = 1: weight sum and union)
// or pass 2 (out[k]: the frame's level-0 Gaussian as 3 f32 planes, its
// normalised mask (f32) and support (u8), plane = pitch * H elements).
struct Remap16Args {
  int32_t W, H;
  int32_t window_ok;
  int32_t K;
  int32_t accumulate;
  int32_t first;
  float inv_count;       // 1 / N, the mask where the weight sum is <= 1e-12
  float* norm;
  uint8_t* uni;
  int64_t pitch;
  FrameIn f[kMaxBatch];  // src.px: u16 samples, src.pitch in bytes
  LevelPlanes out[kMaxBatch];
};
cudaError_t launch_remap16_weights(const Remap16Args& a, int border, cudaStream_t s);
// Standalone u16 remap: dst holds dst_ch u16 samples per pixel.
cudaError_t launch_remap16(const RemapArgs& a, cudaStream_t s);
// 1 x 1 stacks: acc += G0_k * m_k over the batch (a.out planes, a.K frames).
cudaError_t launch_blend_single_level(float* acc, int64_t acc_plane, const Remap16Args& a, cudaStream_t s);
cudaError_t launch_lap0(const Lap0Args& a, int border, cudaStream_t s);
// hybrid-pyramid-contrast (src/stack/pipeline.zig:177-236): winners of the
// hardmask method over a batch of frames' pass-2 planes (first batch: best
// weights start at -inf), the plain Laplacian pyramids of the soft and hard
// images and their merge (src/fuse/pyramid.zig:271-301, 418-488).
cudaError_t launch_winners(const FramePlanes* planes, int K, float* best, uint32_t* hard, int first, int w, int h,
                           int64_t pitch, cudaStream_t s);
// Level 0 of a pyramid: interleaved RGB(A) u8 samples (bytes per pixel 3 or
// 4) to three f32 planes (fillRgbBase of an image without alpha).
cudaError_t launch_rgb_to_planes(const uint8_t* src, int64_t src_pitch, int px_bytes, float* dst, int64_t plane,
                                 int64_t pitch, int w, int h, cudaStream_t s);
// Plain clamped five-tap REDUCE of three planes (reduceRgbRowsSequential,
// src/fuse/pyramid.zig:950-995, 1725-1746).
cudaError_t launch_reduce_plain(const float* src, int64_t splane, int64_t spitch, int sw, int sh, float* dst,
                                int64_t dplane, int64_t dpitch, int dw, int dh, cudaStream_t s);
struct MergeArgs {
  int32_t wp, hp, wc, hc;       // level l and level l + 1 sizes
  int64_t pitch_p, pitch_c, plane_p, plane_c;
  int32_t exact_expand;         // max(wp, hp) <= 512
  int32_t mixed;                // level inside the hard range: soft + (hard - soft) * mix
  float mix;
  const float* soft_p;          // Gaussians of the soft / hard images at level l and l + 1
  const float* hard_p;
  const float* soft_c;
  const float* hard_c;
  float* acc;                   // merged Laplacian of level l (pitch_p, plane_p)
};
cudaError_t launch_merge_level(const MergeArgs& a, cudaStream_t s);
// The top level: the Gaussians themselves, mixed when inside the hard range.
cudaError_t launch_merge_top(const float* soft, const float* hard, float* acc, int64_t plane, int64_t pitch, int w,
                             int h, int mixed, float mix, cudaStream_t s);

// acc0 = A_w / N where N > 1e-12, else A_u * inv_count (acc0 written over A_w).
cudaError_t launch_finalize0(float* acc, const float* au, const float* norm, int64_t plane, int64_t pitch, int w,
                             int h, float inv_count, cudaStream_t s);
cudaError_t launch_level0(const LevelArgs& a, int storage, cudaStream_t s);
cudaError_t launch_level(const LevelArgs& a, int storage, cudaStream_t s);
cudaError_t launch_collapse(const CollapseArgs& a, cudaStream_t s);
// Split pyramid: the image half of a level step for the batch's frames, one
// frame per CTA (grid.z = K): Gaussian REDUCE to level l + 1 (slots out[k],
// or gtop[k] at the top) and the Laplacian of level l into lap[k] (FP32 at
// level 0, the storage type above); level 0 reads the remapped RGBA planes
// in0[k].rgba.
cudaError_t launch_img_level(const LevelArgs& a, int storage, cudaStream_t s);
// Level-0 blend of all frames of a split-pyramid stack (device tables of
// each frame's level-0 Laplacian and weight planes) fused with every frame's
// level-0 mask REDUCE: acc = sum over frames, in order, of lap[k] x (w_k /
// weight sum) (1 / N where the sum is <= 1e-12), written over acc, and
// mask1[k] (level-1 size wn x hn, row pitch pitch_n, in out_storage) the
// REDUCE of those normalised masks with the union support sm (row pitch
// `pitch`), as launch_mask_reduce forms it; the weight planes are only read.
// lap null: the masks alone (acc untouched), the level-0 mask pyramid step
// of a FUSED stack.
cudaError_t launch_blend0_reduce(float* acc, int64_t plane, int64_t pitch, int w, int h, const float* norm,
                                 const uint8_t* sm, const float* const* lap, const float* const* wgt,
                                 void* const* mask1, int64_t pitch_n, int wn, int hn, int frames, float inv_count,
                                 int out_storage, cudaStream_t s);
// out[i] = w[i] / n[i] as the level-0 blend divides (the refinement from
// the correctly rounded reciprocal), on device arrays of `count` floats.
cudaError_t launch_normalise_check(const float* w, const float* n, float* out, size_t count, cudaStream_t s);
// The same for a level l >= 1 of a split-pyramid stack: acc = sum over
// frames, in order, of lap[k] x mask[k] (both in `storage`; 3 Laplacian
// planes of `plane` samples), and mask_next[k] the REDUCE of mask[k] with
// the level's mask support sm, as launch_blend and launch_mask_reduce give
// them (level l + 1: wn x hn, row pitch pitch_n, in out_storage).
cudaError_t launch_blend_reduce(float* acc, int64_t plane, int64_t pitch, int w, int h, const uint8_t* sm,
                                const void* const* lap, const void* const* mask, void* const* mask_next,
                                int64_t pitch_n, int wn, int hn, int frames, int storage, int out_storage,
                                cudaStream_t s);
// Tiles a level needs (64 x 32 each) for launch_blend_reduce to fill the GPU
// better than the per-frame launches: below it the mask REDUCE and the blend
// of the level run apart, with every frame in the grid.
static constexpr int64_t kBlendReduceMinTiles = 1184;
// acc = sum over frames k, in order, of lap[k] (3 planes of `plane`) times
// mask[k] (both in storage T: 0 f32, 1 f16, 2 bf16), written over acc.
cudaError_t launch_blend(float* acc, int64_t plane, int64_t pitch, int w, int h, const void* const* lap,
                         const void* const* mask, int frames, int storage, cudaStream_t s);
// acc[c] += contrib[k][c] for k = 0 .. K-1 in order (w x h level, plane stride `plane`).
cudaError_t launch_sum_contrib(float* acc, int64_t plane, int64_t pitch, int w, int h, const float* contrib, int K,
                               cudaStream_t s);
cudaError_t launch_mask_support(const MaskSupportArgs& a, cudaStream_t s);
cudaError_t launch_remap(const RemapArgs& a, cudaStream_t s);
cudaError_t launch_quantize(const float* acc, int64_t plane, int64_t pitch, int w, int h, uint8_t* out,
                            int64_t out_pitch, float* base, int64_t base_pitch, int out16, cudaStream_t s);

// Small-level tail of the split pyramid: the levels whose sides are both at
// most kTailSide, from level T >= 1 up to the top (at most kMaxTail steps),
// in three launches instead of four per level.
static constexpr int kTailSide = 64;
static constexpr int kMaxTail = 8;

// Pass 1: the image half of the level steps T .. T + steps - 1 of a batch
// (lv[i] as launch_img_level takes it for level T + i), one frame per CTA,
// the levels one after another inside the CTA.
struct ImgTailArgs {
  int32_t steps;
  int32_t pad;
  LevelArgs lv[kMaxTail];
};
cudaError_t launch_img_tail(const ImgTailArgs& a, int frames, int storage, cudaStream_t s);

struct TailLevel {
  int32_t w, h;
  int64_t pitch;   // elements (bytes for u8 planes)
  float* acc;      // accumulator, 3 planes
  int64_t plane;   // elements per accumulator plane
};
// Pass 2 over levels T .. L-1 of a LAPS / FUSED stack.  tab: the stack's
// frame table (per level l: N Laplacian pointers, the top level's Gaussians,
// then N mask pointers; level-l masks in the level storage, the top's f32).
struct BlendTailArgs {
  int32_t first;             // T (>= 1)
  int32_t levels;            // L
  int32_t frames;            // N
  int32_t storage;           // level storage of levels T .. L-2
  const void* const* tab;
  const uint8_t* sm_first;   // union mask support of level T
  uint32_t* counter;         // zero before the blend launch; the launch leaves it zero
  TailLevel lv[kMaxTail + 1];  // levels T .. L-1
};
// Each frame's masks of levels T+1 .. L-1 (one frame per CTA; the mask
// support of those levels is formed in shared memory).
cudaError_t launch_mask_tail(const BlendTailArgs& a, cudaStream_t s);
// The blend of levels T .. L-1 over every frame in order, then (last CTA to
// finish) the collapse of those levels down to level T.
cudaError_t launch_blend_tail(const BlendTailArgs& a, cudaStream_t s);

// Synthetic stacks (synth.cu).
void synth_pose(uint64_t seed, int scene, uint32_t width, uint32_t height, uint32_t frame, uint32_t frame_count,
                fs_pose* p);
int synth_render(uint64_t seed, int scene, uint32_t width, uint32_t height, uint32_t frame, uint32_t frame_count,
                 void* dev_out, size_t out_stride, fs_pose* pose_out, cudaStream_t stream, const char** why);

// Normaliser of the no-wrap expand (shared by host checks and the kernels).
FS_HD float exact_expand_divisor(int x, int y, int sw, int sh) {
  const int j = x >> 1, q = y >> 1;
  const bool xe = (x & 1) == 0, ye = (y & 1) == 0;
  if (sh == 1) {
    if (sw == 1) return ye ? (xe ? 36.f : 24.f) : (xe ? 6.f : 4.f);
    if (j < sw - 1) return ye ? (xe ? (j == 0 ? 42.f : 48.f) : 48.f) : (xe ? (j == 0 ? 7.f : 8.f) : 8.f);
    return ye ? (xe ? 49.f : 28.f) : (xe ? 7.f : 4.f);
  }
  if (q < sh - 1) {
    if (sw == 1 || j == sw - 1) return ye ? (xe ? (q == 0 ? 49.f : 56.f) : (q == 0 ? 28.f : 32.f)) : (xe ? 14.f : 8.f);
    if (ye) return xe ? (q == 0 ? (j == 0 ? 49.f : 56.f) : (j == 0 ? 56.f : 64.f)) : (q == 0 ? 56.f : 64.f);
    return xe ? (j == 0 ? 14.f : 16.f) : 16.f;
  }
  if (sw == 1) return ye ? (xe ? 42.f : 28.f) : (xe ? 6.f : 4.f);
  if (j < sw - 1) return ye ? (xe ? (j == 0 ? 49.f : 56.f) : 56.f) : (xe ? (j == 0 ? 7.f : 8.f) : 8.f);
  return ye ? (xe ? 49.f : 28.f) : (xe ? 7.f : 4.f);
}

}  // namespace fs
