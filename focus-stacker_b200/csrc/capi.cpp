// C ABI of libfocuscuda.so: contexts, stacks (two-pass pyramid-contrast
// fusion), remap-only and synthetic-input entry points.
//
// A stack holds on the device: the weight sums and union support of pass 1
// (level-0 planes), the mask-support pyramid, the FP32 accumulator pyramid,
// K per-frame level slots for pass 2, and (when the HBM budget allows) the
// frames themselves, so pass 2 does not need them again from the host.  The
// host side only composes per-frame transforms (FP64) and sequences launches
// on one stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "../../include/focuscuda.h"
#include "fs_common.h"
#include "fs_host.h"
#include "fusion_kernels.cuh"
#include "jpeg.h"

using namespace fs;

namespace {

struct KernelTiming {
  const char* name;
  cudaEvent_t start, stop;
};

}  // namespace

struct fs_ctx {
  int device = 0;
  uint64_t budget = 0;
  uint64_t held = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy = nullptr;
  cudaStream_t idle = nullptr;  // given no work: frees of finished stacks take effect at once
  // level schedule of the split-pyramid stacks begun from now on (0: defaults)
  uint32_t fuse_min_tiles = 0;  // levels l >= 1 of at least this many tiles blend and REDUCE in one pass
  uint32_t tail_side = 0;       // levels with both sides at most this go to the small-level tail
  std::string err;
  mutable std::mutex mu;
  bool timing = false;
  std::vector<KernelTiming> timings;
  uint64_t launches = 0;
  // Stream-ordered memory pool of the device, shared by every context of
  // the process on it: buffers are allocated and freed on a context's
  // streams (no device-wide synchronisation) and freed memory stays cached in
  // the pool for later stacks of any context until fs_ctx_trim.  The budget
  // counts live buffers (`held`); the cache never exceeds the peak of live
  // buffers of all contexts together.
  cudaMemPool_t mempool = nullptr;
  // Live stacks: fs_destroy releases their device memory and detaches them,
  // so that a later fs_stack_destroy of a stack that outlived its context
  // only frees the host record.
  std::set<fs_stack*> stacks;
  // JPEG decoding workspace, grown to the largest file decoded so far: the
  // parsed tables, the unstuffed entropy-coded bytes and interval bounds,
  // coefficients, component planes and the decode status flag.
  struct JpegWork {
    void* tables = nullptr;
    uint8_t* data = nullptr;
    size_t data_cap = 0;
    uint32_t* seg = nullptr;
    size_t seg_cap = 0;
    int16_t* coef = nullptr;
    size_t coef_cap = 0;
    uint8_t* planes = nullptr;
    size_t planes_cap = 0;
    int* status = nullptr;
  } jpeg;
};

namespace {

struct Alloc {
  void* p = nullptr;
  size_t bytes = 0;
};

int set_err(fs_ctx* ctx, int code, const std::string& msg) {
  if (ctx) {
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->err = msg;
  }
  return code;
}

int cuda_err(fs_ctx* ctx, cudaError_t e, const char* what) {
  return set_err(ctx, FS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// The device's shared pool (created once; cached memory is kept until trimmed).
cudaMemPool_t device_pool(int device) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> g(mu);
  auto it = pools.find(device);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  // reuse memory only once its free has completed: a stream of one context
  // must never be made to wait for another context's queued work
  int no = 0;
  cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
  pools[device] = pool;
  return pool;
}

// Release the pool's cached (freed) memory; waits for the context's streams.
void pool_trim(fs_ctx* ctx) {
  cudaStreamSynchronize(ctx->stream);
  cudaStreamSynchronize(ctx->copy);
  if (ctx->mempool) cudaMemPoolTrimTo(ctx->mempool, 0);
}

// Buffer from the device pool, ordered on `on` (the compute stream by
// default; frame buffers that the copy stream fills first are allocated on
// the copy stream, so that uploads never wait for queued kernels).
int dev_alloc(fs_ctx* ctx, size_t bytes, void** out, cudaStream_t on = nullptr) {
  if (bytes == 0) bytes = 16;
  if (ctx->held + bytes > ctx->budget)
    return set_err(ctx, FS_ERR_BUDGET, "device memory budget exceeded (" + std::to_string(ctx->held + bytes) +
                                           " > " + std::to_string(ctx->budget) + " bytes)");
  cudaError_t e = cudaMallocFromPoolAsync(out, bytes, ctx->mempool, on ? on : ctx->stream);
  if (e == cudaErrorMemoryAllocation && ctx->mempool) {
    // the pool keeps freed memory for reuse; when a request finds none that
    // fits, give back what it holds unused (completed frees only) and retry
    cudaGetLastError();
    cudaMemPoolTrimTo(ctx->mempool, 0);
    e = cudaMallocFromPoolAsync(out, bytes, ctx->mempool, on ? on : ctx->stream);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, FS_ERR_OOM, std::string("device allocation failed: ") + cudaGetErrorString(e));
  }
  ctx->held += bytes;
  return FS_OK;
}

// Stream-ordered free; callers make sure the copy stream is done with the
// buffer (stacks synchronise both streams before releasing).
void dev_free(fs_ctx* ctx, void* p, size_t bytes, cudaStream_t on = nullptr) {
  if (!p) return;
  cudaFreeAsync(p, on ? on : ctx->stream);
  if (bytes == 0) bytes = 16;
  ctx->held -= std::min<uint64_t>(ctx->held, bytes);
}

// Launch wrapper: counts launches and optionally brackets them with events
// on the launching stream.
template <typename F>
cudaError_t timed(fs_ctx* ctx, const char* name, F&& launch) {
  KernelTiming t = {name, nullptr, nullptr};
  if (ctx->timing) {
    cudaEventCreate(&t.start);
    cudaEventCreate(&t.stop);
    cudaEventRecord(t.start, ctx->stream);
  }
  cudaError_t e = launch();
  ctx->launches += 1;
  if (ctx->timing) {
    cudaEventRecord(t.stop, ctx->stream);
    ctx->timings.push_back(t);
  }
  return e;
}

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

}  // namespace

// ===================================================================== stack
// Pass-2 source of a stack, chosen at fs_stack_begin from the HBM budget:
//  CACHE     pass 1 keeps every remapped frame (RGBA u32) and its weight on
//            the device; pass 2 reads them (the reference's cached path,
//            src/stack/pipeline.zig:454-457, 515-560);
//  RESIDENT  frames stay on the device and pass 2 remaps them again;
//  REFETCH   frames are only staged; pass 2 asks the caller for them again
//            and remaps them (src/stack/pipeline.zig:561-597).
//  LAPS      pass 1 also builds each frame's Gaussian/Laplacian pyramid (it
//            does not depend on the weight sum) and keeps its Laplacians and
//            weight; pass 2 is then only the mask pyramid and the blend.  Same
//            operations, so the same bytes as the other modes; it moves most
//            of pass 2 into pass 1, which overlaps the frame uploads.
//  FUSED     the split pyramid with level 0 fused into pass 1: one kernel
//            remaps, weights, reduces to level 1 and sums lap0 * w over the
//            frames (divided by the weight sum once it is complete), so no
//            level-0 Laplacian or remapped frame is kept: 9-10 bytes per
//            frame-pixel instead of LAPS's 21.  Level 0 rounds in another
//            order (within a few ulp of the accumulator).  The mode for
//            stacks whose LAPS planes do not fit.
enum Pass2Mode { P2_CACHE = 0, P2_RESIDENT = 1, P2_REFETCH = 2, P2_LAPS = 3, P2_FUSED = 4 };

struct fs_stack {
  fs_ctx* ctx = nullptr;
  fs_stack_desc d;
  fs_rect roi;
  uint32_t W = 0, H = 0, L = 0, K = 1, border = 2;
  bool aligned = false;
  int storage = FS_STORAGE_F32;
  Pass2Mode mode = P2_CACHE;
  std::vector<uint32_t> lw, lh;
  std::vector<int64_t> pitch;  // per level, elements (f32) == bytes (u8)
  float* norm = nullptr;
  uint8_t* uni = nullptr;
  std::vector<uint8_t*> sm;    // mask support, level l (sm[0] == uni)
  std::vector<float*> acc;     // per level, 3 planes
  std::vector<std::vector<LevelPlanes>> slot;  // [k][l], l = 1 .. L-2
  std::vector<FramePlanes> cache;              // CACHE: per frame
  std::vector<FramePlanes> p2;                 // RESIDENT / REFETCH / LAPS: per batch slot (K)
  std::vector<LevelPlanes> slot0;              // 16-bit frames: level-0 planes per batch slot (K)
  uint32_t bps = 1;                            // bytes per sample (1: u8, 2: u16)
  int method = FS_METHOD_PYRAMID_CONTRAST;     // fs_stack_set_method
  float hybrid_mix = 0.35f;                    // hybrid: weight of the hard image's levels
  float* best = nullptr;                       // hybrid: per pixel the winning weight
  uint32_t* hard = nullptr;                    // hybrid: per pixel the winning frame's RGBA word
  std::vector<float*> wplane;                  // LAPS / FUSED: per frame, its weight (level 0)
  std::vector<std::vector<void*>> lap;         // LAPS / FUSED: per frame, Laplacian of levels 0 .. L-2 (level 0:
                                               // f32, LAPS only; above: the storage type)
  float* au = nullptr;                         // FUSED: sum of level-0 Laplacians where the weight sum <= 1e-12
  std::vector<float*> gtop;                    // LAPS / FUSED: per frame, Gaussian of the top level
  std::vector<std::vector<void*>> mplane;      // LAPS / FUSED: per frame, mask of levels 1 .. L-2 (storage type)
  std::vector<float*> mtop;                    // LAPS / FUSED: per frame, mask of the top level (f32)
  std::vector<const float*> tab_host;          // LAPS / FUSED: per level, Laplacian then mask pointers of all frames
  const float** tab = nullptr;                 // the same table on the device
  uint8_t* out_dev = nullptr;
  std::vector<Alloc> allocs;
  struct Frame {
    const uint8_t* px = nullptr;  // device pointer (owned or borrowed)
    int64_t pitch = 0;
    bool owned = false;
    bool resident = true;         // false: transient staging copy, pass 2 refetches it
    int slot = -1;                // staging buffer of a transient copy
    fs_pose pose;
  };
  std::vector<Frame> frames;
  std::vector<uint8_t*> staging;  // transient frame buffers (K)
  int64_t frame_pitch = 0;        // pitch of owned frame copies
  size_t frame_bytes = 0;
  size_t pass1_done = 0;          // frames whose pass 1 has been launched
  bool finished = false;
  cudaEvent_t copy_done = nullptr;
  cudaEvent_t done = nullptr;     // recorded after the output copy of fs_stack_finish_async
  // the exact-sample queue of a pass-1 / pass-2 remap batch (8-bit frames)
  uint32_t* exact_n = nullptr;
  uint64_t* exact_q = nullptr;
  uint32_t exact_cap = 0;
  std::vector<cudaEvent_t> slot_done;  // per staging buffer: the remap that last read it
  float* base_out = nullptr;      // optional device buffer for the collapsed base (RGB f32)
  uint32_t fp_level = 0;          // first level run one frame per CTA (none: >= L - 1)
  uint32_t frame_total = 0;       // frames of the whole stack when this one holds a shard (0: its own)
  int phase = 0;                  // 0 adding frames, 1 pass 1 done, 2 blended
  float* contrib = nullptr;       // per-frame blend contributions of those levels
  float* contrib_top = nullptr;   // and of the top level
  int64_t base_pitch = 0;         // elements
  // Batches: the stack's buffers are carved from its lane's arena (shared by
  // the lane's stacks, which run one after another) instead of the pool.
  uint8_t* arena = nullptr;
  size_t arena_size = 0, arena_used = 0;
  // LAPS / FUSED: first level of the small-level tail (0: none) and the
  // blend-tail launch's ticket (zero between launches)
  uint32_t tail = 0;
  uint32_t* tail_counter = nullptr;
  int64_t fuse_min_tiles = kBlendReduceMinTiles;  // the context's schedule at begin
  bool tail_folded = false;  // pass 2 has added the tail levels' EXPANDs into acc[tail]
};

namespace {

uint32_t in_channels(const fs_stack* s) { return s->d.channels; }

// Free a stack's device memory and events and cut it from its context (the
// context's streams must be idle).
void detach_stack(fs_stack* s) {
  if (!s->ctx) return;
  for (auto& a : s->allocs) dev_free(s->ctx, a.p, a.bytes);
  s->allocs.clear();
  if (s->copy_done) cudaEventDestroy(s->copy_done);
  if (s->done) cudaEventDestroy(s->done);
  for (cudaEvent_t& ev : s->slot_done)
    if (ev) cudaEventDestroy(ev), ev = nullptr;
  s->slot_done.clear();
  s->copy_done = nullptr;
  s->done = nullptr;
  s->ctx = nullptr;
}

// Arena pieces start on 256-byte boundaries, as pool allocations do.
constexpr size_t kArenaAlign = 256;

// pooled: from the context's pool even for an arena stack (buffers whose
// contents are written once, at begin, and must survive the lane's other
// stacks).
int stack_alloc(fs_stack* s, size_t bytes, void** out, cudaStream_t on = nullptr, bool pooled = false) {
  if (s->arena && !pooled) {
    const size_t at = round_up((int64_t)s->arena_used, (int64_t)kArenaAlign);
    const size_t n = bytes == 0 ? 16 : bytes;
    if (at + n > s->arena_size)
      return set_err(s->ctx, FS_ERR_BUDGET, "stack needs more than its lane arena (" + std::to_string(at + n) +
                                                " > " + std::to_string(s->arena_size) + " bytes)");
    *out = s->arena + at;
    s->arena_used = at + n;
    return FS_OK;
  }
  int rc = dev_alloc(s->ctx, bytes, out, on);
  if (rc == FS_OK) s->allocs.push_back({*out, bytes == 0 ? 16 : bytes});
  return rc;
}

bool build_frame_in(fs_stack* s, const fs_stack::Frame& fr, FrameIn* fi, std::string* why) {
  std::memset(fi, 0, sizeof(*fi));
  fi->src.px = fr.px;
  fi->src.pitch = fr.pitch;
  fi->src.w = (int32_t)s->d.src_width;
  fi->src.h = (int32_t)s->d.src_height;
  fi->src.ch = (int32_t)in_channels(s);
  if (s->aligned) {
    fi->warp.kind = WARP_ALIGNED;
    return true;
  }
  // the remap addresses its taps with 32-bit offsets
  if (s->bps == 1 && (uint64_t)fr.pitch * s->d.src_height >= (1ull << 32)) {
    *why = "source frames of 4 GiB or more (row stride x height) are not supported";
    return false;
  }
  const char* w = nullptr;
  if (!compose_warp(fr.pose, s->d.src_width, s->d.src_height, s->roi, &fi->warp, &w)) {
    *why = w ? w : "invalid pose";
    return false;
  }
  return true;
}

// remap + weights for frames [begin, end): pass 1 (accumulate, and keep
// the planes in CACHE / LAPS mode) or pass 2 of RESIDENT / REFETCH (planes
// into the batch slots, no accumulation).
int launch_remap_weights_batch(fs_stack* s, const std::vector<fs_stack::Frame>& frames, size_t begin, size_t end,
                               bool pass1) {
  RemapWeightArgs a;
  std::memset(&a, 0, sizeof(a));
  a.W = (int32_t)s->W;
  a.H = (int32_t)s->H;
  a.window_ok = (s->W >= s->d.contrast_window && s->H >= s->d.contrast_window) ? 1 : 0;
  a.K = (int32_t)(end - begin);
  a.accumulate = pass1 ? 1 : 0;
  a.first = begin == 0 ? 1 : 0;
  a.norm = s->norm;
  a.uni = s->uni;
  a.pitch = s->pitch[0];
  a.exact_q = s->exact_q;
  a.exact_n = s->exact_n;
  a.exact_cap = s->exact_cap;
  for (size_t k = begin; k < end; ++k) {
    std::string why;
    if (!build_frame_in(s, frames[k], &a.f[k - begin], &why)) return set_err(s->ctx, FS_ERR_INVALID, why);
    if (pass1) {
      // the weights are formed from the remapped words: modes that keep no
      // planes in pass 1 remap into the (still unused) pass-2 batch slots
      if (s->mode == P2_CACHE) a.out[k - begin] = s->cache[k];
      else if (s->mode == P2_LAPS) a.out[k - begin] = FramePlanes{s->p2[k - begin].rgba, s->wplane[k]};
      else a.out[k - begin] = FramePlanes{s->p2[k - begin].rgba, nullptr};
    } else {
      a.out[k - begin] = s->p2[k - begin];
    }
  }
  cudaError_t e = timed(s->ctx, pass1 ? "pass1" : "remap_weights",
                        [&] { return launch_remap_weights(a, (int)s->border, s->ctx->stream); });
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "remap/weights launch");
  // the remap of the tiles, its exact samples, then the weights
  s->ctx->launches += a.exact_q ? 2 : 1;
  return FS_OK;
}

// Geometry of the step from level l to l + 1 (the fields every level kernel
// reads), frames of the batch left to the caller.
void level_geometry(const fs_stack* s, uint32_t l, LevelArgs* a) {
  a->level = (int32_t)l;
  a->wl = (int32_t)s->lw[l];
  a->hl = (int32_t)s->lh[l];
  a->pitch_l = s->pitch[l];
  a->exact_expand = std::max(s->lw[l], s->lh[l]) <= kExactExpandMaxDim ? 1 : 0;
  a->sm_l = s->sm[l];
  a->acc_l = s->acc[l];
  a->acc_plane_l = s->pitch[l] * s->lh[l];
  if (l + 1 < s->L) {
    a->wn = (int32_t)s->lw[l + 1];
    a->hn = (int32_t)s->lh[l + 1];
    a->pitch_n = s->pitch[l + 1];
    a->acc_n = s->acc[l + 1];
    a->acc_plane_n = s->pitch[l + 1] * s->lh[l + 1];
  } else {
    a->wn = a->hn = 1;
    a->pitch_n = 32;
  }
}

// 16-bit frames [begin, end): pass 1 (weight sum and union) or pass 2
// (level-0 planes into the batch slots).
int launch_remap16_batch(fs_stack* s, const std::vector<fs_stack::Frame>& frames, size_t begin, size_t end,
                         bool pass1, float inv_count) {
  Remap16Args a;
  std::memset(&a, 0, sizeof(a));
  a.W = (int32_t)s->W;
  a.H = (int32_t)s->H;
  a.window_ok = (s->W >= s->d.contrast_window && s->H >= s->d.contrast_window) ? 1 : 0;
  a.K = (int32_t)(end - begin);
  a.accumulate = pass1 ? 1 : 0;
  a.first = begin == 0 ? 1 : 0;
  a.inv_count = inv_count;
  a.norm = s->norm;
  a.uni = s->uni;
  a.pitch = s->pitch[0];
  for (size_t k = begin; k < end; ++k) {
    std::string why;
    if (!build_frame_in(s, frames[k], &a.f[k - begin], &why)) return set_err(s->ctx, FS_ERR_INVALID, why);
    if (!pass1) a.out[k - begin] = s->slot0[k - begin];
  }
  cudaError_t e = timed(s->ctx, pass1 ? "pass1" : "remap_weights",
                        [&] { return launch_remap16_weights(a, (int)s->border, s->ctx->stream); });
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "16-bit remap/weights launch");
  if (!pass1 && s->L == 1) {
    e = timed(s->ctx, "level0", [&] {
      return launch_blend_single_level(s->acc[0], s->pitch[0] * s->lh[0], a, s->ctx->stream);
    });
    if (e != cudaSuccess) return cuda_err(s->ctx, e, "single-level blend");
  }
  return FS_OK;
}

// FUSED pass 1, level 0 of frames [begin, end): remap, weights (weight sum
// and union), level-1 Gaussian into the batch slots, A_w += lap0 * w.
int launch_lap0_batch(fs_stack* s, size_t begin, size_t end) {
  Lap0Args a;
  std::memset(&a, 0, sizeof(a));
  a.W = (int32_t)s->W;
  a.H = (int32_t)s->H;
  a.window_ok = (s->W >= s->d.contrast_window && s->H >= s->d.contrast_window) ? 1 : 0;
  a.K = (int32_t)(end - begin);
  a.first = begin == 0 ? 1 : 0;
  a.exact_expand = std::max(s->lw[0], s->lh[0]) <= kExactExpandMaxDim ? 1 : 0;
  a.wn = (int32_t)s->lw[1];
  a.hn = (int32_t)s->lh[1];
  a.storage = s->storage;
  a.pitch = s->pitch[0];
  a.pitch_n = s->pitch[1];
  a.plane = s->pitch[0] * s->lh[0];
  a.norm = s->norm;
  a.uni = s->uni;
  a.aw = s->acc[0];
  a.au = s->au;
  a.best = s->best;
  a.hard = s->hard;
  // the remap of the batch into its RGBA slots, then the fused level 0 from them
  RemapWeightArgs r;
  std::memset(&r, 0, sizeof(r));
  r.W = a.W;
  r.H = a.H;
  r.K = a.K;
  r.pitch = s->pitch[0];
  r.exact_q = s->exact_q;
  r.exact_n = s->exact_n;
  r.exact_cap = s->exact_cap;
  for (size_t k = begin; k < end; ++k) {
    std::string why;
    if (!build_frame_in(s, s->frames[k], &r.f[k - begin], &why)) return set_err(s->ctx, FS_ERR_INVALID, why);
    r.out[k - begin] = FramePlanes{s->p2[k - begin].rgba, nullptr};
    a.rgba[k - begin] = s->p2[k - begin].rgba;
    a.w[k - begin] = s->wplane[k];
    a.g1[k - begin] = s->slot[k - begin][1];
  }
  cudaError_t e = timed(s->ctx, "pass1", [&] { return launch_remap_tiles(r, s->ctx->stream); });
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "remap launch");
  if (r.exact_q) s->ctx->launches += 1;  // and its exact samples
  e = timed(s->ctx, "pass1", [&] { return launch_lap0(a, (int)s->border, s->ctx->stream); });
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "fused pass-1 launch");
  return FS_OK;
}

// LAPS / FUSED pass 1: the Gaussian / Laplacian pyramid of frames [begin,
// end), one frame per CTA, from their remapped RGBA in the batch slots (LAPS,
// from level 0) or their level-1 Gaussians (FUSED, from level 1).
int launch_image_pyramid(fs_stack* s, size_t begin, size_t end) {
  LevelArgs a;
  std::memset(&a, 0, sizeof(a));
  a.levels = (int32_t)s->L;
  a.K = (int32_t)(end - begin);
  const uint32_t tail = s->tail ? s->tail : s->L;  // levels from here on: one tail launch
  ImgTailArgs t;
  t.steps = 0;
  t.pad = 0;
  for (uint32_t l = s->mode == P2_FUSED ? 1 : 0; l + 1 < s->L; ++l) {
    level_geometry(s, l, &a);
    for (size_t k = 0; k < (size_t)a.K; ++k) {
      if (l == 0) a.in0[k] = s->p2[k];
      else a.in[k] = s->slot[k][l];
      a.out[k] = l + 1 < s->L - 1 ? s->slot[k][l + 1] : LevelPlanes{};
      a.lap[k] = s->lap[begin + k][l];
      a.gtop[k] = s->gtop[begin + k];
    }
    if (l >= tail) {
      t.lv[t.steps++] = a;
      continue;
    }
    cudaError_t e = timed(s->ctx, "image", [&] { return launch_img_level(a, s->storage, s->ctx->stream); });
    if (e != cudaSuccess) return cuda_err(s->ctx, e, "image pyramid launch");
  }
  if (t.steps > 0) {
    cudaError_t e = timed(s->ctx, "image", [&] { return launch_img_tail(t, a.K, s->storage, s->ctx->stream); });
    if (e != cudaSuccess) return cuda_err(s->ctx, e, "image pyramid tail launch");
  }
  return FS_OK;
}

// Pass 1 runs in batches of K frames as they arrive; the last frames of the
// stack go in smaller batches (each of the last kTailFrames on arrival), so
// that little pass-1 work is left once the last frame is in.
constexpr size_t kTailFrames = 2;

int run_pending_pass1(fs_stack* s, bool flush) {
  for (;;) {
    const size_t pending = s->frames.size() - s->pass1_done;
    const size_t to_come = s->d.frame_count - s->frames.size();
    if (!(pending >= s->K || (pending > 0 && (flush || to_come <= kTailFrames)))) break;
    size_t begin = s->pass1_done, end = std::min(s->frames.size(), begin + s->K);
    int rc = s->mode == P2_FUSED ? launch_lap0_batch(s, begin, end)
             : s->bps == 2       ? launch_remap16_batch(s, s->frames, begin, end, true, 0.0f)
                                 : launch_remap_weights_batch(s, s->frames, begin, end, true);
    if (rc != FS_OK) return rc;
    // the staging buffers of these frames are free for reuse after this remap
    for (size_t f = begin; f < end; ++f) {
      const int slot = s->frames[f].slot;
      if (slot < 0) continue;
      cudaError_t e = cudaEventRecord(s->slot_done[slot], s->ctx->stream);
      if (e != cudaSuccess) return cuda_err(s->ctx, e, "pass-1 event");
    }
    if (s->mode == P2_LAPS && s->best) {
      // hybrid: the hardmask winners of the batch, from its pass-1 planes
      FramePlanes pl[kMaxBatch];
      for (size_t k = begin; k < end; ++k) pl[k - begin] = FramePlanes{s->p2[k - begin].rgba, s->wplane[k]};
      cudaError_t e = timed(s->ctx, "winners", [&] {
        return launch_winners(pl, (int)(end - begin), s->best, s->hard, begin == 0 ? 1 : 0, (int)s->W, (int)s->H,
                              s->pitch[0], s->ctx->stream);
      });
      if (e != cudaSuccess) return cuda_err(s->ctx, e, "winners");
    }
    if ((s->mode == P2_LAPS || s->mode == P2_FUSED) && (rc = launch_image_pyramid(s, begin, end)) != FS_OK)
      return rc;
    s->pass1_done = end;
  }
  return FS_OK;
}

// ------------------------------------------------------------------- JPEG
void jpeg_release(fs_ctx* ctx) {
  fs_ctx::JpegWork& j = ctx->jpeg;
  dev_free(ctx, j.tables, sizeof(jpeg::Tables));
  dev_free(ctx, j.data, j.data_cap);
  dev_free(ctx, j.seg, j.seg_cap * 8);
  dev_free(ctx, j.coef, j.coef_cap * 2);
  dev_free(ctx, j.planes, j.planes_cap);
  dev_free(ctx, j.status, 16);
  j = fs_ctx::JpegWork();
}

// Grow a workspace buffer to `need` (elements of `esz` bytes), ordered on the
// context's stream.
template <typename T>
int jpeg_grow(fs_ctx* ctx, T** buf, size_t* cap, size_t need, size_t esz) {
  if (*buf && *cap >= need) return FS_OK;
  dev_free(ctx, *buf, *cap * esz);
  *buf = nullptr;
  *cap = 0;
  void* p;
  const int rc = dev_alloc(ctx, need * esz, &p);
  if (rc != FS_OK) return rc;
  *buf = (T*)p;
  *cap = need;
  return FS_OK;
}

// Decode a JPEG file into device RGB u8 (row pitch in bytes), queued on the
// context's stream.  expect_w / expect_h != 0: the file must have that size.
// The host buffer may be reused once this returns.
int jpeg_decode(fs_ctx* ctx, const void* data, size_t len, uint8_t* d_dst, int64_t dst_pitch, uint32_t expect_w,
                uint32_t expect_h) {
  jpeg::Parsed P;
  std::string why;
  if (!jpeg::parse((const uint8_t*)data, len, &P, &why)) return set_err(ctx, FS_ERR_UNSUPPORTED, "JPEG: " + why);
  if (expect_w && (P.width != expect_w || P.height != expect_h))
    return set_err(ctx, FS_ERR_MISMATCH, "JPEG frame size differs from the stack's");
  fs_ctx::JpegWork& j = ctx->jpeg;
  int rc;
  if (!j.tables) {
    if ((rc = dev_alloc(ctx, sizeof(jpeg::Tables), &j.tables)) != FS_OK) return rc;
    void* p;
    if ((rc = dev_alloc(ctx, 16, &p)) != FS_OK) return rc;
    j.status = (int*)p;
    if (cudaMemsetAsync(j.status, 0, sizeof(int), ctx->stream) != cudaSuccess)
      return cuda_err(ctx, cudaGetLastError(), "JPEG status");
  }
  const size_t ncoef = jpeg::coef_count(P.t);
  if ((rc = jpeg_grow(ctx, &j.coef, &j.coef_cap, ncoef, 2)) != FS_OK) return rc;
  if ((rc = jpeg_grow(ctx, &j.planes, &j.planes_cap, ncoef, 1)) != FS_OK) return rc;  // one sample per coefficient
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(j.tables, &P.t, sizeof(jpeg::Tables), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(j.coef, 0, ncoef * 2, st);
  if (e != cudaSuccess) return cuda_err(ctx, e, "JPEG upload");
  const int nseg = (int)P.seg_begin.size();
  if (nseg > 1) {
    // restart intervals: entropy decoding on the GPU, one thread per interval
    if ((rc = jpeg_grow(ctx, &j.data, &j.data_cap, std::max<size_t>(P.data.size(), 16), 1)) != FS_OK) return rc;
    if ((rc = jpeg_grow(ctx, &j.seg, &j.seg_cap, (size_t)nseg, 8)) != FS_OK) return rc;
    std::vector<uint32_t> seg(P.seg_begin);
    seg.insert(seg.end(), P.seg_end.begin(), P.seg_end.end());
    e = cudaMemcpyAsync(j.data, P.data.data(), P.data.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(j.seg, seg.data(), seg.size() * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = timed(ctx, "jpeg", [&] {
        return jpeg::launch_entropy((const jpeg::Tables*)j.tables, j.data, j.seg, j.seg + nseg, nseg, j.coef, j.status,
                                    st);
      });
    if (e != cudaSuccess) return cuda_err(ctx, e, "JPEG entropy decoding");
  } else {
    // one interval: a sequential bitstream, decoded on the host
    std::vector<int16_t> coef(ncoef, 0);
    if (!jpeg::decode_interval(P.t, P.data.data(), 0, (uint32_t)P.data.size(), 0,
                               (int64_t)P.t.mcus_x * P.t.mcus_y, coef.data()))
      return set_err(ctx, FS_ERR_INVALID, "JPEG: corrupt entropy-coded data");
    e = cudaMemcpyAsync(j.coef, coef.data(), ncoef * 2, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // `coef` goes out of scope
    if (e != cudaSuccess) return cuda_err(ctx, e, "JPEG coefficient upload");
  }
  e = timed(ctx, "jpeg", [&] {
    return jpeg::launch_idct_color((const jpeg::Tables*)j.tables, P.t, j.coef, j.planes, P.width, P.height, d_dst,
                                   dst_pitch, st);
  });
  if (e != cudaSuccess) return cuda_err(ctx, e, "JPEG inverse DCT / colour");
  return FS_OK;
}

// Read and clear the JPEG status flag (waits for the stream).
int jpeg_status(fs_ctx* ctx) {
  if (!ctx->jpeg.status) return FS_OK;
  int v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, ctx->jpeg.status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->jpeg.status, 0, sizeof(int), ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_err(ctx, e, "JPEG status");
  return v ? set_err(ctx, FS_ERR_INVALID, "JPEG: corrupt entropy-coded data") : FS_OK;
}

}  // namespace

extern "C" {

int fs_api_version(void) { return FS_API_VERSION; }

const char* fs_status_string(int status) {
  switch (status) {
    case FS_OK: return "ok";
    case FS_ERR_INVALID: return "invalid argument";
    case FS_ERR_OOM: return "out of memory";
    case FS_ERR_BUDGET: return "device memory budget exceeded";
    case FS_ERR_CUDA: return "CUDA error";
    case FS_ERR_TIMEOUT: return "device wait timed out";
    case FS_ERR_STATE: return "call out of order";
    case FS_ERR_MISMATCH: return "frame does not match the stack";
    case FS_ERR_UNSUPPORTED: return "unsupported";
    case FS_ERR_NO_DEVICE: return "no usable CUDA device";
    default: return "unknown status";
  }
}

void fs_pose_default(fs_pose* p) {
  std::memset(p, 0, sizeof(*p));
  p->base_hfov_degrees = 50.0;
}

int fs_create(int device, uint64_t hbm_budget_bytes, fs_ctx** out) {
  if (!out) return FS_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) {
    cudaGetLastError();
    return FS_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) {
    cudaGetLastError();
    return FS_ERR_NO_DEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) return FS_ERR_NO_DEVICE;
  fs_ctx* c = new fs_ctx();
  c->device = device;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  c->budget = hbm_budget_bytes ? hbm_budget_bytes : (uint64_t)(free_b / 2);
  c->mempool = device_pool(device);
  if (!c->mempool || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->idle, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return FS_ERR_CUDA;
  }
  *out = c;
  return FS_OK;
}

void fs_destroy(fs_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStreamSynchronize(ctx->copy);
  for (fs_stack* s : ctx->stacks) detach_stack(s);
  ctx->stacks.clear();
  jpeg_release(ctx);
  pool_trim(ctx);
  for (auto& t : ctx->timings) {
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->copy) cudaStreamDestroy(ctx->copy);
  if (ctx->idle) cudaStreamDestroy(ctx->idle);
  delete ctx;
}

const char* fs_last_error(const fs_ctx* ctx) {
  if (!ctx) return "no context";
  return ctx->err.c_str();
}

uint64_t fs_ctx_device_bytes(const fs_ctx* ctx) { return ctx ? ctx->held : 0; }

uint64_t fs_ctx_budget(const fs_ctx* ctx) { return ctx ? ctx->budget : 0; }

int fs_ctx_set_budget(fs_ctx* ctx, uint64_t hbm_budget_bytes) {
  if (!ctx || hbm_budget_bytes == 0) return FS_ERR_INVALID;
  ctx->budget = hbm_budget_bytes;
  return FS_OK;
}

int fs_ctx_set_level_schedule(fs_ctx* ctx, uint32_t fuse_min_tiles, uint32_t tail_side) {
  if (!ctx) return FS_ERR_INVALID;
  if (tail_side > (uint32_t)kTailSide) return set_err(ctx, FS_ERR_INVALID, "tail side above the tail kernels' 64");
  ctx->fuse_min_tiles = fuse_min_tiles;
  ctx->tail_side = tail_side;
  return FS_OK;
}

int fs_ctx_reserve(fs_ctx* ctx, uint64_t bytes) {
  if (!ctx) return FS_ERR_INVALID;
  if (bytes == 0) return FS_OK;
  cudaSetDevice(ctx->device);
  void* p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, ctx->mempool, ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, FS_ERR_OOM, std::string("reserve: ") + cudaGetErrorString(e));
  }
  e = cudaFreeAsync(p, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? FS_OK : cuda_err(ctx, e, "reserve");
}

int fs_ctx_trim(fs_ctx* ctx) {
  if (!ctx) return FS_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  pool_trim(ctx);
  return FS_OK;
}

int fs_check_normalise(fs_ctx* ctx, const float* w, const float* n, float* out, size_t count) {
  if (!ctx || (count && (!w || !n || !out))) return FS_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaError_t e = launch_normalise_check(w, n, out, count, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? FS_OK : cuda_err(ctx, e, "normalise check");
}

int fs_ctx_stream(const fs_ctx* ctx, void** stream) {
  if (!ctx || !stream) return FS_ERR_INVALID;
  *stream = (void*)ctx->stream;
  return FS_OK;
}

int fs_ctx_set_kernel_timing(fs_ctx* ctx, int enable) {
  if (!ctx) return FS_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& t : ctx->timings) {
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  ctx->timings.clear();
  ctx->timing = enable != 0;
  return FS_OK;
}

int fs_ctx_kernel_stats(fs_ctx* ctx, const char* kernel, uint64_t* launches, double* total_ms) {
  if (!ctx || !kernel) return FS_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_err(ctx, e, "synchronize");
  uint64_t n = 0;
  double ms = 0.0;
  for (auto& t : ctx->timings) {
    if (std::strcmp(t.name, kernel) != 0) continue;
    float v = 0.f;
    cudaEventElapsedTime(&v, t.start, t.stop);
    ms += v;
    ++n;
  }
  if (launches) *launches = n;
  if (total_ms) *total_ms = ms;
  return FS_OK;
}

uint64_t fs_ctx_launch_count(const fs_ctx* ctx) { return ctx ? ctx->launches : 0; }

int fs_ctx_synchronize(fs_ctx* ctx) {
  if (!ctx) return FS_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_err(ctx, e, "synchronize");
  return FS_OK;
}

// ---------------------------------------------------------------- pose utils
int fs_compute_roi(const fs_pose* poses, const uint32_t* widths, const uint32_t* heights, const uint8_t* active,
                   size_t n, fs_rect* out, int* has_roi) {
  if (!poses || !widths || !heights || !out || !has_roi) return FS_ERR_INVALID;
  fs_rect r = {0, 0, 0, 0};
  bool ok = compute_roi(poses, widths, heights, active, n, &r);
  *has_roi = ok ? 1 : 0;
  *out = r;
  return FS_OK;
}

int fs_inverse_map_points(const fs_pose* pose, uint32_t width, uint32_t height, size_t n, const double* xy,
                          double* out_xy) {
  if (!pose || (!xy && n) || (!out_xy && n)) return FS_ERR_INVALID;
  for (size_t i = 0; i < n; ++i)
    inverse_map_point_f64(*pose, width, height, xy[2 * i], xy[2 * i + 1], &out_xy[2 * i], &out_xy[2 * i + 1]);
  return FS_OK;
}

int fs_forward_map_points(const fs_pose* pose, uint32_t width, uint32_t height, size_t n, const double* xy,
                          double* out_xy) {
  if (!pose || (!xy && n) || (!out_xy && n)) return FS_ERR_INVALID;
  for (size_t i = 0; i < n; ++i)
    forward_map_point(*pose, width, height, xy[2 * i], xy[2 * i + 1], &out_xy[2 * i], &out_xy[2 * i + 1]);
  return FS_OK;
}

// Host evaluation of the kernels' no-wrap expand normaliser (for checks of
// the closed form against the reference's sequential SKIPSM expand).
float fs_exact_expand_divisor(int x, int y, int src_w, int src_h) { return exact_expand_divisor(x, y, src_w, src_h); }

// ------------------------------------------------------------------- remap
static int remap_impl(fs_ctx* ctx, const void* src, size_t src_stride, uint32_t width, uint32_t height,
                      uint32_t channels, const fs_pose* pose, const fs_rect* roi, void* dst, size_t dst_stride,
                      bool device, int bytes_per_sample = 1) {
  if (!ctx || !src || !dst || !pose) return set_err(ctx, FS_ERR_INVALID, "null argument");
  if (channels != 1 && channels != 3) return set_err(ctx, FS_ERR_UNSUPPORTED, "remap supports 1 or 3 channels");
  if (width == 0 || height == 0) return set_err(ctx, FS_ERR_INVALID, "empty frame");
  fs_rect r = roi ? *roi : fs_rect{0, 0, (int32_t)width, (int32_t)height};
  if (r.right <= r.left || r.bottom <= r.top) return set_err(ctx, FS_ERR_INVALID, "empty roi");
  uint32_t ow = (uint32_t)(r.right - r.left), oh = (uint32_t)(r.bottom - r.top);
  if (src_stride < (size_t)width * channels * bytes_per_sample ||
      dst_stride < (size_t)ow * (channels + 1) * bytes_per_sample)
    return set_err(ctx, FS_ERR_INVALID, "row stride too small");
  cudaSetDevice(ctx->device);
  RemapArgs a;
  std::memset(&a, 0, sizeof(a));
  const char* why = nullptr;
  if (!compose_warp(*pose, width, height, r, &a.f.warp, &why)) return set_err(ctx, FS_ERR_INVALID, why);
  a.W = (int32_t)ow;
  a.H = (int32_t)oh;
  a.dst_ch = (int32_t)channels + 1;
  a.f.src.w = (int32_t)width;
  a.f.src.h = (int32_t)height;
  a.f.src.ch = (int32_t)channels;
  void *dsrc = nullptr, *ddst = nullptr;
  size_t sbytes = src_stride * height, dbytes = dst_stride * oh;
  if (device) {
    dsrc = const_cast<void*>(src);
    ddst = dst;
  } else {
    int rc = dev_alloc(ctx, sbytes, &dsrc);
    if (rc != FS_OK) return rc;
    rc = dev_alloc(ctx, dbytes, &ddst);
    if (rc != FS_OK) {
      dev_free(ctx, dsrc, sbytes);
      return rc;
    }
    cudaMemcpyAsync(dsrc, src, sbytes, cudaMemcpyHostToDevice, ctx->stream);
  }
  a.f.src.px = (const uint8_t*)dsrc;
  a.f.src.pitch = (int64_t)src_stride;
  a.dst = (uint8_t*)ddst;
  a.dst_pitch = (int64_t)dst_stride;
  cudaError_t e = timed(ctx, "remap", [&] {
    return bytes_per_sample == 2 ? launch_remap16(a, ctx->stream) : launch_remap(a, ctx->stream);
  });
  if (e == cudaSuccess && !device) e = cudaMemcpyAsync(dst, ddst, dbytes, cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
  if (!device) {
    dev_free(ctx, dsrc, sbytes);
    dev_free(ctx, ddst, dbytes);
  }
  if (e != cudaSuccess) return cuda_err(ctx, e, "remap");
  if (e2 != cudaSuccess) return cuda_err(ctx, e2, "remap");
  return FS_OK;
}

int fs_remap_frame(fs_ctx* ctx, const void* src, size_t src_stride, uint32_t width, uint32_t height,
                   uint32_t channels, const fs_pose* pose, const fs_rect* roi, void* dst, size_t dst_stride) {
  return remap_impl(ctx, src, src_stride, width, height, channels, pose, roi, dst, dst_stride, false);
}

int fs_remap_frame16(fs_ctx* ctx, const void* src, size_t src_stride, uint32_t width, uint32_t height,
                     uint32_t channels, const fs_pose* pose, const fs_rect* roi, void* dst, size_t dst_stride) {
  return remap_impl(ctx, src, src_stride, width, height, channels, pose, roi, dst, dst_stride, false, 2);
}

int fs_remap_frame16_device(fs_ctx* ctx, const void* src, size_t src_stride, uint32_t width, uint32_t height,
                            uint32_t channels, const fs_pose* pose, const fs_rect* roi, void* dst,
                            size_t dst_stride) {
  return remap_impl(ctx, src, src_stride, width, height, channels, pose, roi, dst, dst_stride, true, 2);
}

int fs_remap_frame_device(fs_ctx* ctx, const void* src, size_t src_stride, uint32_t width, uint32_t height,
                          uint32_t channels, const fs_pose* pose, const fs_rect* roi, void* dst, size_t dst_stride) {
  return remap_impl(ctx, src, src_stride, width, height, channels, pose, roi, dst, dst_stride, true);
}

// ------------------------------------------------------------------- stacks
namespace {

// Validation of a stack description (null when valid; the status in *code).
const char* check_desc(const fs_stack_desc& d, int* code) {
  *code = FS_ERR_INVALID;
  if (d.sample_bits != 8 && d.sample_bits != 16) return "sample_bits must be 8 or 16";
  if (d.sample_bits == 16 && d.level_storage != FS_STORAGE_F32) {
    *code = FS_ERR_UNSUPPORTED;
    return "16-bit samples need FP32 level storage (FP16 tops out at 65504, BF16 keeps 8 bits)";
  }
  if (d.src_width == 0 || d.src_height == 0 || d.frame_count == 0) return "empty stack";
  if (d.contrast_window < 3 || (d.contrast_window & 1) == 0) return "contrast window must be odd and >= 3";
  if (d.contrast_window > 2 * kMaxBorder + 1) {
    *code = FS_ERR_UNSUPPORTED;
    return "contrast window larger than 15";
  }
  if (d.level_storage != FS_STORAGE_F32 && d.level_storage != FS_STORAGE_F16 && d.level_storage != FS_STORAGE_BF16)
    return "unknown level storage";
  const bool aligned = d.input_is_aligned != 0;
  if (aligned ? (d.channels != 3 && d.channels != 4) : d.channels != 3)
    return "channels must be 3 (RGB source) or 3/4 (aligned RGB/RGBA)";
  if (!aligned && d.has_roi && (d.roi.right <= d.roi.left || d.roi.bottom <= d.roi.top)) return "empty roi";
  return nullptr;
}

// Geometry and device-memory plan of a stack: what fs_stack_begin allocates
// (fixed state, per-frame or per-batch planes) and what add_frame adds later
// (upload staging or kept frames).
struct StackPlan {
  fs_rect roi;
  uint32_t W, H, L, K;
  std::vector<uint32_t> lw, lh;
  std::vector<int64_t> pitch;
  size_t fixed = 0;          // weight sum, union, supports, accumulators, level slots, output
  size_t planes = 0;         // pass-1 planes of one frame (RGBA + weight)
  size_t frame_bytes = 0;    // one device copy of a source frame
  int64_t frame_pitch = 0;
  size_t staging_slots = 0;  // frame buffers of the two-batch upload ring
  uint32_t fp_level = 0;     // first level l >= 1 run one frame per CTA (L - 1: none)
  size_t contrib = 0, contrib_top = 0;  // bytes of the contribution buffers
  size_t laps_frame = 0;                // LAPS: weight, Laplacians, top Gaussian and masks of one frame
  size_t fused_frame = 0;               // FUSED: the same without the level-0 Laplacian
  size_t fused_fixed = 0;               // FUSED: the level-0 Laplacian sum of the fallback pixels
  uint32_t exact_cap = 0;               // entries of the exact-sample queue (0: none)
};

// The exact-sample queue of a remap batch: kExactPerTile entries per tile and
// frame of a batch (8-bit remapped frames only: aligned frames are not
// sampled, 16-bit frames take the exact path in their own kernels), after a
// 16-byte counter.
uint32_t exact_queue_cap(const StackPlan& p, const fs_stack_desc& d) {
  if (d.input_is_aligned || d.sample_bits == 16) return 0;
  const uint64_t tiles = (uint64_t)((p.W + kTileW - 1) / kTileW) * ((p.H + kTileH - 1) / kTileH);
  return (uint32_t)std::min<uint64_t>(tiles * p.K * kExactPerTile, 1u << 30);
}
size_t exact_queue_bytes(uint32_t cap) { return cap ? 16 + (size_t)cap * 8 : 0; }

// Levels with fewer 64x32 tiles than this run one frame per CTA (grid.z = K)
// and add the frames' contributions in order afterwards: a small level has
// too few tiles to fill the GPU when each CTA walks all K frames.
constexpr uint32_t kFrameParallelTiles = 592;

StackPlan plan_stack(const fs_stack_desc& d) {
  StackPlan p;
  const bool aligned = d.input_is_aligned != 0;
  p.roi = d.has_roi && !aligned ? d.roi : fs_rect{0, 0, (int32_t)d.src_width, (int32_t)d.src_height};
  p.W = (uint32_t)(p.roi.right - p.roi.left);
  p.H = (uint32_t)(p.roi.bottom - p.roi.top);
  p.L = level_count(p.W, p.H);
  const uint32_t k = d.frames_per_batch ? d.frames_per_batch : 8;
  p.K = std::max(1u, std::min<uint32_t>(std::min<uint32_t>(k, (uint32_t)kMaxBatch), d.frame_count));
  uint32_t w = p.W, h = p.H;
  for (uint32_t l = 0; l < p.L; ++l) {
    p.lw.push_back(w);
    p.lh.push_back(h);
    p.pitch.push_back(round_up(w, 32));
    w = next_level_size(w);
    h = next_level_size(h);
  }
  const size_t esz = d.level_storage == FS_STORAGE_F32 ? 4 : 2;
  const size_t bps = d.sample_bits == 16 ? 2 : 1;
  const size_t n0 = (size_t)p.pitch[0] * p.H;
  p.fixed = n0 * 4 + n0;                                                            // weight sum, union
  for (uint32_t l = 1; l < p.L; ++l) p.fixed += (size_t)p.pitch[l] * p.lh[l];       // mask support
  for (uint32_t l = 0; l < p.L; ++l) p.fixed += (size_t)p.pitch[l] * p.lh[l] * 12;  // accumulators
  for (uint32_t l = 1; l + 1 < p.L; ++l) p.fixed += p.K * ((size_t)p.pitch[l] * p.lh[l] * (esz * 4 + 1));
  p.fixed += (size_t)p.W * p.H * 3 * bps;  // output
  p.exact_cap = exact_queue_cap(p, d);
  p.fixed += exact_queue_bytes(p.exact_cap);
  // per frame (cache) or batch slot: remapped RGBA + weight; 16-bit frames:
  // level-0 Gaussian (3 f32 planes), normalised mask (f32) and support (u8)
  p.planes = bps == 2 ? n0 * 17 : n0 * 8;
  p.frame_pitch = round_up((int64_t)d.src_width * d.channels * (int64_t)bps, 16);
  p.frame_bytes = (size_t)p.frame_pitch * d.src_height;
  p.staging_slots = std::min<size_t>(2 * (size_t)p.K, d.frame_count);
  p.fp_level = p.L > 1 ? p.L - 1 : 1;
  if (p.K > 1) {
    for (uint32_t l = 1; l + 1 < p.L; ++l) {
      const uint32_t tiles = ((p.lw[l] + kTileW - 1) / kTileW) * ((p.lh[l] + kTileH - 1) / kTileH);
      if (tiles < kFrameParallelTiles) {
        p.fp_level = l;
        break;
      }
    }
  }
  if (p.L >= 3 && bps == 1) {
    p.fused_frame = n0 * 4;                                                                      // weight
    for (uint32_t l = 1; l + 1 < p.L; ++l) p.fused_frame += (size_t)p.pitch[l] * p.lh[l] * 3 * esz;  // Laplacians
    p.fused_frame += (size_t)p.pitch[p.L - 1] * p.lh[p.L - 1] * 12;  // top Gaussian
    for (uint32_t l = 1; l + 1 < p.L; ++l) p.fused_frame += (size_t)p.pitch[l] * p.lh[l] * esz;  // masks
    p.fused_frame += (size_t)p.pitch[p.L - 1] * p.lh[p.L - 1] * 4;  // top mask
    p.fused_fixed = n0 * 12;
    p.laps_frame = p.fused_frame + n0 * 12;  // and the level-0 Laplacian (f32)
  }
  if (p.fp_level + 1 < p.L) {
    p.contrib = (size_t)p.K * 3 * p.pitch[p.fp_level] * p.lh[p.fp_level] * 4;
    p.contrib_top = (size_t)p.K * 3 * p.pitch[p.L - 1] * p.lh[p.L - 1] * 4;
    p.fixed += p.contrib + p.contrib_top;
  }
  return p;
}

// Device bytes of a stack over its life in pass-2 mode `mode`; the upload
// staging ring counts when frames come from host memory.
uint64_t plan_bytes(const StackPlan& p, uint32_t frames, Pass2Mode mode, bool host_frames) {
  const uint64_t staging = host_frames ? (uint64_t)p.frame_bytes * p.staging_slots : 0;
  // split pyramid: the frame table and, after it, the small-level tail's counter
  const uint64_t table = 16;
  switch (mode) {
    case P2_LAPS:
      return p.fixed + (uint64_t)p.planes / 2 * p.K + ((uint64_t)p.laps_frame + 2 * p.L * sizeof(float*)) * frames +
             table + staging;
    case P2_FUSED:
      return p.fixed + p.fused_fixed + (uint64_t)p.planes / 2 * p.K +
             ((uint64_t)p.fused_frame + 2 * p.L * sizeof(float*)) * frames + table + staging;
    case P2_CACHE: return p.fixed + (uint64_t)p.planes * frames + staging;
    case P2_RESIDENT: return p.fixed + (uint64_t)p.planes * p.K + (uint64_t)p.frame_bytes * frames;
    default: return p.fixed + (uint64_t)p.planes * p.K + staging;
  }
}

// Pass-2 mode for `available` device bytes: cache the pass-1 planes when they
// fit, else keep the frames, else refetch them.
Pass2Mode choose_mode(const StackPlan& p, uint32_t frames, uint64_t available, bool host_frames, bool wide) {
  if (p.laps_frame && plan_bytes(p, frames, P2_LAPS, host_frames) <= available) return P2_LAPS;
  if (p.fused_frame && plan_bytes(p, frames, P2_FUSED, host_frames) <= available) return P2_FUSED;
  if (!wide && plan_bytes(p, frames, P2_CACHE, host_frames) <= available) return P2_CACHE;
  if (plan_bytes(p, frames, P2_RESIDENT, host_frames) <= available) return P2_RESIDENT;
  return P2_REFETCH;
}

}  // namespace

// forced_mode >= 0: pass-2 mode chosen by the caller (batches plan it);
// arena: device memory the stack's buffers are carved from (batches).
static int begin_impl(fs_ctx* ctx, const fs_stack_desc* desc, fs_stack** out, int forced_mode,
                      uint8_t* arena = nullptr, size_t arena_size = 0) {
  if (!ctx || !desc || !out) return set_err(ctx, FS_ERR_INVALID, "null argument");
  *out = nullptr;
  const fs_stack_desc& d = *desc;
  int code = FS_OK;
  if (const char* why = check_desc(d, &code)) return set_err(ctx, code, why);
  cudaSetDevice(ctx->device);
  const StackPlan plan = plan_stack(d);
  fs_stack* s = new fs_stack();
  s->ctx = ctx;
  ctx->stacks.insert(s);
  s->d = d;
  s->roi = plan.roi;
  s->aligned = d.input_is_aligned != 0;
  s->storage = d.level_storage;
  s->bps = d.sample_bits == 16 ? 2 : 1;
  s->W = plan.W;
  s->H = plan.H;
  s->L = plan.L;
  s->border = d.contrast_window / 2;
  s->K = plan.K;
  s->lw = plan.lw;
  s->lh = plan.lh;
  s->pitch = plan.pitch;
  s->arena = arena;
  s->arena_size = arena ? arena_size : 0;
  if (ctx->fuse_min_tiles) s->fuse_min_tiles = ctx->fuse_min_tiles;
  auto fail = [&](int rc) {
    fs_stack_destroy(s);
    return rc;
  };
  int rc;
  void* p;
  const size_t n0 = (size_t)s->pitch[0] * s->H;
  if ((rc = stack_alloc(s, n0 * 4, &p)) != FS_OK) return fail(rc);
  s->norm = (float*)p;
  if ((rc = stack_alloc(s, n0, &p)) != FS_OK) return fail(rc);
  s->uni = (uint8_t*)p;
  if (plan.exact_cap) {
    if ((rc = stack_alloc(s, exact_queue_bytes(plan.exact_cap), &p)) != FS_OK) return fail(rc);
    s->exact_n = (uint32_t*)p;
    s->exact_q = (uint64_t*)((uint8_t*)p + 16);
    s->exact_cap = plan.exact_cap;
  }
  s->sm.push_back(s->uni);
  for (uint32_t l = 1; l < s->L; ++l) {
    if ((rc = stack_alloc(s, (size_t)s->pitch[l] * s->lh[l], &p)) != FS_OK) return fail(rc);
    s->sm.push_back((uint8_t*)p);
  }
  for (uint32_t l = 0; l < s->L; ++l) {
    if ((rc = stack_alloc(s, (size_t)s->pitch[l] * s->lh[l] * 3 * 4, &p)) != FS_OK) return fail(rc);
    s->acc.push_back((float*)p);
  }
  const size_t esz = s->storage == FS_STORAGE_F32 ? 4 : 2;
  s->slot.assign(s->K, std::vector<LevelPlanes>(s->L));
  for (uint32_t kk = 0; kk < s->K; ++kk) {
    for (uint32_t l = 1; l + 1 < s->L; ++l) {
      const size_t plane = (size_t)s->pitch[l] * s->lh[l];
      LevelPlanes lp;
      if ((rc = stack_alloc(s, plane * esz * 4 + plane, &p)) != FS_OK) return fail(rc);
      lp.g = p;
      lp.m = (uint8_t*)p + plane * esz * 3;
      lp.s = (uint8_t*)p + plane * esz * 4;
      lp.plane = (int64_t)plane;
      s->slot[kk][l] = lp;
    }
  }
  if ((rc = stack_alloc(s, (size_t)s->W * s->H * 3 * s->bps, &p)) != FS_OK) return fail(rc);
  s->out_dev = (uint8_t*)p;
  s->fp_level = plan.fp_level;
  if (plan.contrib) {
    if ((rc = stack_alloc(s, plan.contrib, &p)) != FS_OK) return fail(rc);
    s->contrib = (float*)p;
    if ((rc = stack_alloc(s, plan.contrib_top, &p)) != FS_OK) return fail(rc);
    s->contrib_top = (float*)p;
  }
  // pass-2 source from what the budget leaves (this stack's fixed state is
  // already held and part of every mode's bytes)
  s->frame_pitch = plan.frame_pitch;
  s->frame_bytes = plan.frame_bytes;
  const uint64_t in_use = ctx->held;
  const uint64_t available = ctx->budget + plan.fixed > in_use ? ctx->budget + plan.fixed - in_use : 0;
  s->mode = forced_mode >= 0 ? (Pass2Mode)forced_mode
                             : choose_mode(plan, d.frame_count, available, true, d.sample_bits == 16);
  const size_t planes_bytes = plan.planes;
  if (s->mode == P2_LAPS || s->mode == P2_FUSED) {
    const bool laps = s->mode == P2_LAPS;
    // remapped RGBA of the batch's frames, read by the level-0 image step
    // (LAPS) or the fused level-0 kernel (FUSED)
    for (uint32_t kk = 0; kk < s->K; ++kk) {
      if ((rc = stack_alloc(s, n0 * 4, &p)) != FS_OK) return fail(rc);
      s->p2.push_back(FramePlanes{(uint32_t*)p, nullptr});
    }
    if (!laps) {
      if ((rc = stack_alloc(s, plan.fused_fixed, &p)) != FS_OK) return fail(rc);
      s->au = (float*)p;
    }
    for (uint32_t f = 0; f < d.frame_count; ++f) {
      if ((rc = stack_alloc(s, laps ? plan.laps_frame : plan.fused_frame, &p)) != FS_OK) return fail(rc);
      uint8_t* q = (uint8_t*)p;
      s->wplane.push_back((float*)q);
      q += n0 * 4;
      std::vector<void*> lv(1, nullptr);  // FUSED: level 0 is blended by the fused pass-1 kernel
      if (laps) {
        lv[0] = q;  // level-0 Laplacian, f32
        q += n0 * 12;
      }
      for (uint32_t l = 1; l + 1 < s->L; ++l) {
        lv.push_back(q);
        q += (size_t)s->pitch[l] * s->lh[l] * 3 * esz;
      }
      s->lap.push_back(lv);
      s->gtop.push_back((float*)q);
      q += (size_t)s->pitch[s->L - 1] * s->lh[s->L - 1] * 12;
      std::vector<void*> mv(s->L, nullptr);
      for (uint32_t l = 1; l + 1 < s->L; ++l) {
        mv[l] = q;
        q += (size_t)s->pitch[l] * s->lh[l] * esz;
      }
      s->mplane.push_back(mv);
      s->mtop.push_back((float*)q);
    }
    // per level: Laplacian (top: Gaussian) then mask (level 0: weight) of every frame
    for (uint32_t l = 0; l < s->L; ++l) {
      for (uint32_t f = 0; f < d.frame_count; ++f)
        s->tab_host.push_back(l + 1 < s->L ? (const float*)s->lap[f][l] : s->gtop[f]);
      for (uint32_t f = 0; f < d.frame_count; ++f)
        s->tab_host.push_back(l == 0 ? s->wplane[f] : l + 1 < s->L ? (const float*)s->mplane[f][l] : s->mtop[f]);
    }
    // the small-level tail: levels T >= 1 whose sides are at most kTailSide
    // (or the context's smaller side), when they make two level steps or more
    const uint32_t tail_side = ctx->tail_side ? ctx->tail_side : (uint32_t)kTailSide;
    for (uint32_t l = 1; l < s->L; ++l) {
      if (std::max(s->lw[l], s->lh[l]) <= tail_side) {
        if (s->L - 1 - l >= 2 && s->L - 1 - l <= (uint32_t)kMaxTail) s->tail = l;
        break;
      }
    }
    const size_t tab_bytes = round_up((int64_t)(s->tab_host.size() * sizeof(float*)), 16);
    if ((rc = stack_alloc(s, tab_bytes + 16, &p, nullptr, true)) != FS_OK) return fail(rc);
    s->tab = (const float**)p;
    s->tail_counter = (uint32_t*)((uint8_t*)p + tab_bytes);
    if (cudaMemcpyAsync(p, s->tab_host.data(), s->tab_host.size() * sizeof(float*), cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess ||
        cudaMemsetAsync(s->tail_counter, 0, 16, ctx->stream) != cudaSuccess)
      return fail(cuda_err(ctx, cudaGetLastError(), "frame table upload"));
  } else if (s->mode == P2_CACHE) {
    for (uint32_t f = 0; f < d.frame_count; ++f) {
      if ((rc = stack_alloc(s, planes_bytes, &p)) != FS_OK) return fail(rc);
      s->cache.push_back(FramePlanes{(uint32_t*)p, (float*)((uint8_t*)p + n0 * 4)});
    }
  } else if (s->bps == 2) {
    // level-0 Gaussian (3 f32 planes), normalised mask and support per batch slot
    for (uint32_t kk = 0; kk < s->K; ++kk) {
      if ((rc = stack_alloc(s, planes_bytes, &p)) != FS_OK) return fail(rc);
      s->slot0.push_back(LevelPlanes{p, (uint8_t*)p + n0 * 12, (uint8_t*)p + n0 * 16, (int64_t)n0});
    }
  } else {
    for (uint32_t kk = 0; kk < s->K; ++kk) {
      if ((rc = stack_alloc(s, planes_bytes, &p)) != FS_OK) return fail(rc);
      s->p2.push_back(FramePlanes{(uint32_t*)p, (float*)((uint8_t*)p + n0 * 4)});
    }
  }
  cudaEventCreateWithFlags(&s->copy_done, cudaEventDisableTiming);
  *out = s;
  return FS_OK;
}

int fs_stack_begin(fs_ctx* ctx, const fs_stack_desc* desc, fs_stack** out) { return begin_impl(ctx, desc, out, -1); }

int fs_stack_begin_mode(fs_ctx* ctx, const fs_stack_desc* desc, int pass2_mode, fs_stack** out) {
  if (pass2_mode < -1 || pass2_mode > P2_FUSED) return set_err(ctx, FS_ERR_INVALID, "unknown pass-2 mode");
  if (desc && desc->sample_bits == 16 && (pass2_mode == P2_CACHE || pass2_mode >= P2_LAPS))
    return set_err(ctx, FS_ERR_UNSUPPORTED, "16-bit stacks run the resident or refetch mode");
  if (desc && pass2_mode >= P2_LAPS && plan_stack(*desc).laps_frame == 0)
    return set_err(ctx, FS_ERR_UNSUPPORTED, "the laps and fused modes need at least 3 pyramid levels (8-bit samples)");
  return begin_impl(ctx, desc, out, pass2_mode);
}

// wait_copy: return only once a host frame's upload has completed (the
// caller may reuse its buffer); without it the upload is only queued.
static int add_frame_impl(fs_stack* s, const void* pixels, size_t row_stride, const fs_pose* pose, bool device,
                          bool wait_copy = true) {
  if (!s || !pixels) return FS_ERR_INVALID;
  if (!s->ctx) return FS_ERR_STATE;  // its context was destroyed
  fs_ctx* ctx = s->ctx;
  if (s->finished) return set_err(ctx, FS_ERR_STATE, "stack already finished");
  if (s->frames.size() >= s->d.frame_count) return set_err(ctx, FS_ERR_STATE, "more frames than frame_count");
  if (!s->aligned && !pose) return set_err(ctx, FS_ERR_INVALID, "pose required for source frames");
  const size_t row_bytes = (size_t)s->d.src_width * s->d.channels * s->bps;
  if (row_stride < row_bytes) return set_err(ctx, FS_ERR_MISMATCH, "row stride smaller than the stack's row");
  cudaSetDevice(ctx->device);
  fs_stack::Frame fr;
  if (pose) fr.pose = *pose; else fs_pose_default(&fr.pose);
  if (device) {
    fr.px = (const uint8_t*)pixels;
    fr.pitch = (int64_t)row_stride;
  } else {
    uint8_t* buf = nullptr;
    if (s->mode == P2_RESIDENT) {
      // kept for pass 2
      void* p;
      int rc = stack_alloc(s, s->frame_bytes, &p, ctx->copy);
      if (rc != FS_OK) return rc;
      buf = (uint8_t*)p;
      fr.owned = true;
    } else {
      // staged for pass 1 only: two batches of buffers, so that frames of
      // the next batch upload while pass 1 of the current one runs
      const size_t nslots = 2 * (size_t)s->K;
      const size_t slot = s->frames.size() % nslots;
      while (s->staging.size() <= slot) {
        void* p;
        int rc = stack_alloc(s, s->frame_bytes, &p, ctx->copy);
        if (rc != FS_OK) return rc;
        s->staging.push_back((uint8_t*)p);
        cudaEvent_t ev;
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        s->slot_done.push_back(ev);
      }
      if (s->frames.size() >= nslots) {
        // the remap of the frame 2K back read this buffer: the upload waits for it
        cudaError_t e = cudaStreamWaitEvent(ctx->copy, s->slot_done[slot], 0);
        if (e != cudaSuccess) return cuda_err(ctx, e, "staging reuse");
      }
      buf = s->staging[slot];
      fr.resident = false;
      fr.slot = (int)slot;
    }
    // one linear copy when the rows are packed alike (faster than a pitched copy)
    cudaError_t e = row_stride == (size_t)s->frame_pitch
                        ? cudaMemcpyAsync(buf, pixels, row_stride * s->d.src_height, cudaMemcpyHostToDevice, ctx->copy)
                        : cudaMemcpy2DAsync(buf, (size_t)s->frame_pitch, pixels, row_stride, row_bytes,
                                            s->d.src_height, cudaMemcpyHostToDevice, ctx->copy);
    if (e != cudaSuccess) return cuda_err(ctx, e, "frame upload");
    cudaEventRecord(s->copy_done, ctx->copy);
    cudaStreamWaitEvent(ctx->stream, s->copy_done, 0);
    // the caller may reuse its buffer once this returns
    if (wait_copy) {
      e = cudaEventSynchronize(s->copy_done);
      if (e != cudaSuccess) return cuda_err(ctx, e, "frame upload");
    }
    fr.px = buf;
    fr.pitch = s->frame_pitch;
  }
  s->frames.push_back(fr);
  return run_pending_pass1(s, s->frames.size() == s->d.frame_count);
}

int fs_jpeg_info(const void* data, size_t len, uint32_t* width, uint32_t* height) {
  if (!data || !width || !height) return FS_ERR_INVALID;
  jpeg::Parsed P;
  std::string why;
  if (!jpeg::parse((const uint8_t*)data, len, &P, &why)) return FS_ERR_UNSUPPORTED;
  *width = P.width;
  *height = P.height;
  return FS_OK;
}

int fs_decode_jpeg(fs_ctx* ctx, const void* data, size_t len, void* dst, size_t dst_stride, int device_dst) {
  if (!ctx || !data || !dst) return set_err(ctx, FS_ERR_INVALID, "null argument");
  uint32_t w = 0, h = 0;
  if (fs_jpeg_info(data, len, &w, &h) != FS_OK) {
    jpeg::Parsed P;
    std::string why;
    jpeg::parse((const uint8_t*)data, len, &P, &why);
    return set_err(ctx, FS_ERR_UNSUPPORTED, "JPEG: " + why);
  }
  if (dst_stride < (size_t)w * 3) return set_err(ctx, FS_ERR_INVALID, "output stride too small");
  cudaSetDevice(ctx->device);
  void* ddst = dst;
  const size_t bytes = (size_t)w * 3 * h;
  if (!device_dst) {
    int rc = dev_alloc(ctx, bytes, &ddst);
    if (rc != FS_OK) return rc;
  }
  int rc = jpeg_decode(ctx, data, len, (uint8_t*)ddst, device_dst ? (int64_t)dst_stride : (int64_t)w * 3, 0, 0);
  if (rc == FS_OK && !device_dst) {
    cudaError_t e = cudaMemcpy2DAsync(dst, dst_stride, ddst, (size_t)w * 3, (size_t)w * 3, h, cudaMemcpyDeviceToHost,
                                      ctx->stream);
    if (e != cudaSuccess) rc = cuda_err(ctx, e, "JPEG output copy");
  }
  const int st = jpeg_status(ctx);  // waits for the stream
  if (!device_dst) dev_free(ctx, ddst, bytes);
  return rc != FS_OK ? rc : st;
}

// A JPEG frame of the stack: decoded on the device into the frame's staging
// (or resident) buffer, then pass 1 as for fs_stack_add_frame.
int fs_stack_add_frame_jpeg(fs_stack* s, const void* data, size_t len, const fs_pose* pose) {
  if (!s || !data) return FS_ERR_INVALID;
  if (!s->ctx) return FS_ERR_STATE;
  fs_ctx* ctx = s->ctx;
  if (s->finished) return set_err(ctx, FS_ERR_STATE, "stack already finished");
  if (s->frames.size() >= s->d.frame_count) return set_err(ctx, FS_ERR_STATE, "more frames than frame_count");
  if (!s->aligned && !pose) return set_err(ctx, FS_ERR_INVALID, "pose required for source frames");
  if (s->bps != 1 || s->d.channels != 3) return set_err(ctx, FS_ERR_MISMATCH, "JPEG frames are 8-bit RGB");
  cudaSetDevice(ctx->device);
  fs_stack::Frame fr;
  if (pose) fr.pose = *pose; else fs_pose_default(&fr.pose);
  uint8_t* buf = nullptr;
  if (s->mode == P2_RESIDENT) {
    void* p;
    int rc = stack_alloc(s, s->frame_bytes, &p);
    if (rc != FS_OK) return rc;
    buf = (uint8_t*)p;
    fr.owned = true;
  } else {
    const size_t nslots = 2 * (size_t)s->K;
    const size_t slot = s->frames.size() % nslots;
    while (s->staging.size() <= slot) {
      void* p;
      int rc = stack_alloc(s, s->frame_bytes, &p, ctx->copy);
      if (rc != FS_OK) return rc;
      s->staging.push_back((uint8_t*)p);
      cudaEvent_t ev;
      cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      s->slot_done.push_back(ev);
    }
    // the buffer's allocation (and any raw upload into it) is ordered on the
    // copy stream: the decode on the compute stream waits for it
    cudaEventRecord(s->copy_done, ctx->copy);
    cudaStreamWaitEvent(ctx->stream, s->copy_done, 0);
    buf = s->staging[slot];
    fr.resident = false;
    fr.slot = (int)slot;
  }
  int rc = jpeg_decode(ctx, data, len, buf, s->frame_pitch, s->d.src_width, s->d.src_height);
  if (rc != FS_OK) return rc;
  fr.px = buf;
  fr.pitch = s->frame_pitch;
  s->frames.push_back(fr);
  return run_pending_pass1(s, s->frames.size() == s->d.frame_count);
}

int fs_stack_add_frame(fs_stack* stack, const void* pixels, size_t row_stride, const fs_pose* pose) {
  return add_frame_impl(stack, pixels, row_stride, pose, false);
}

int fs_stack_add_frame_async(fs_stack* stack, const void* pixels, size_t row_stride, const fs_pose* pose) {
  return add_frame_impl(stack, pixels, row_stride, pose, false, false);
}

int fs_stack_add_frame_device(fs_stack* stack, const void* dev_pixels, size_t row_stride, const fs_pose* pose) {
  return add_frame_impl(stack, dev_pixels, row_stride, pose, true);
}

static int pass2_impl(fs_stack* s, fs_frame_fetch_cb refetch, void* user, bool fold_tail);
static int collapse_impl(fs_stack* s, void* out, size_t out_stride, bool device_out, bool wait);

// wait: block until the output is written; mark_done: record the stack's
// done event after the output copy (fs_stack_finish_async / fs_stack_wait).
static int finish_impl(fs_stack* s, fs_frame_fetch_cb refetch, void* user, void* out, size_t out_stride,
                       bool device_out, bool wait = true, bool mark_done = false) {
  if (!s || !out) return FS_ERR_INVALID;
  if (!s->ctx) return FS_ERR_STATE;  // its context was destroyed
  fs_ctx* ctx = s->ctx;
  if (s->finished) return set_err(ctx, FS_ERR_STATE, "stack already finished");
  if (s->frames.size() != s->d.frame_count)
    return set_err(ctx, FS_ERR_STATE, "fewer frames added than frame_count");
  if (out_stride < (size_t)s->W * 3 * s->bps) return set_err(ctx, FS_ERR_INVALID, "output stride too small");
  cudaSetDevice(ctx->device);
  int rc;
  if (s->phase < 1) {
    if ((rc = run_pending_pass1(s, true)) != FS_OK) return rc;
    s->phase = 1;
  }
  if (s->phase < 2) {
    if ((rc = pass2_impl(s, refetch, user, true)) != FS_OK) return rc;
    s->phase = 2;
  }
  if ((rc = collapse_impl(s, out, out_stride, device_out, wait)) != FS_OK) return rc;
  if (wait && (rc = jpeg_status(ctx)) != FS_OK) return rc;  // a corrupt JPEG frame of this stack
  if (mark_done) {
    cudaError_t e = s->done ? cudaSuccess : cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(s->done, ctx->stream);
    if (e != cudaSuccess) return cuda_err(ctx, e, "finish event");
  }
  s->finished = true;
  return FS_OK;
}

// Pass 2: mask-support pyramid, accumulators cleared, the blend of every
// frame into them (in the stack's pass-2 mode).  fold_tail: a LAPS / FUSED
// stack with a small-level tail blends its tail levels and collapses them
// into acc[tail] in the same launches (the accumulators above it are then
// spent: the frame-shard phases, which exchange accumulators, pass false).
static int pass2_impl(fs_stack* s, fs_frame_fetch_cb refetch, void* user, bool fold_tail) {
  fs_ctx* ctx = s->ctx;
  int rc;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const bool split = s->mode == P2_LAPS || s->mode == P2_FUSED;
  const uint32_t tail = split && fold_tail && s->tail && !s->frame_total ? s->tail : s->L;
  s->tail_folded = false;
  // mask-support pyramid (frame independent; the tail forms its own levels)
  for (uint32_t l = 0; l + 1 < s->L && l < tail; ++l) {
    MaskSupportArgs m = {s->sm[l], (int32_t)s->lw[l], (int32_t)s->lh[l], s->pitch[l],
                         s->sm[l + 1], (int32_t)s->lw[l + 1], (int32_t)s->lh[l + 1], s->pitch[l + 1]};
    e = timed(ctx, "mask_support", [&] { return launch_mask_support(m, st); });
    if (e != cudaSuccess) return cuda_err(ctx, e, "mask support");
  }
  // (the split-pyramid blends write every accumulator level whole)
  for (uint32_t l = 0; l < s->L && s->mode != P2_LAPS && s->mode != P2_FUSED; ++l) {
    e = cudaMemsetAsync(s->acc[l], 0, (size_t)s->pitch[l] * s->lh[l] * 3 * 4, st);
    if (e != cudaSuccess) return cuda_err(ctx, e, "accumulator clear");
  }
  // pass 2 in batches of K frames; the mask fallback 1/N counts every frame
  // of the stack, also those of other shards
  const size_t N = s->frames.size();
  const float inv_count = 1.0f / (float)(s->frame_total ? s->frame_total : N);
  if (s->mode == P2_LAPS || s->mode == P2_FUSED) {
    if (s->mode == P2_LAPS) {
      // level-0 blend of every frame at once, with each frame's level-0 mask
      // REDUCE to level 1 in the same pass (LAPS needs three levels or more)
      const int out_storage = 2 < s->L ? s->storage : FS_STORAGE_F32;
      e = timed(ctx, "blend0", [&] {
        return launch_blend0_reduce(s->acc[0], s->pitch[0] * s->lh[0], s->pitch[0], (int)s->W, (int)s->H, s->norm,
                                    s->sm[0], s->tab, s->tab + N, (void* const*)(s->tab + 3 * N), s->pitch[1],
                                    (int)s->lw[1], (int)s->lh[1], (int)N, inv_count, out_storage, st);
      });
    } else {
      // level 0: the weighted Laplacian sum of pass 1 divided by the complete
      // weight sum (the 1/N fallback from the plain sum)
      e = timed(ctx, "blend0", [&] {
        return launch_finalize0(s->acc[0], s->au, s->norm, s->pitch[0] * s->lh[0], s->pitch[0], (int)s->W,
                                (int)s->H, inv_count, st);
      });
    }
    if (e != cudaSuccess) return cuda_err(ctx, e, "level-0 blend");
    // the mask pyramid of every frame from level 1 on, level by level (one
    // frame per grid z; level 0's masks come from the level-0 tile kernel)
    auto mask_reduce = [&](uint32_t l) {
      MaskReduceArgs m;
      m.in = (const void* const*)(s->tab + (size_t)l * 2 * N + N);
      m.out = (void* const*)(s->tab + (size_t)(l + 1) * 2 * N + N);
      m.sm = s->sm[l];
      m.wl = (int32_t)s->lw[l];
      m.hl = (int32_t)s->lh[l];
      m.wn = (int32_t)s->lw[l + 1];
      m.hn = (int32_t)s->lh[l + 1];
      m.pitch_l = s->pitch[l];
      m.pitch_n = s->pitch[l + 1];
      const int out_storage = l + 2 < s->L ? s->storage : FS_STORAGE_F32;
      return timed(ctx, "level", [&] { return launch_mask_reduce(m, (int)N, s->storage, out_storage, st); });
    };
    if (s->mode == P2_FUSED && 1 < s->L && 0 < tail) {
      // FUSED level 0: every frame's normalised masks REDUCEd to level 1 (the
      // blend of level 0 happened in pass 1)
      const int out_storage = 2 < s->L ? s->storage : FS_STORAGE_F32;
      e = timed(ctx, "level0", [&] {
        return launch_blend0_reduce(nullptr, s->pitch[0] * s->lh[0], s->pitch[0], (int)s->W, (int)s->H, s->norm,
                                    s->sm[0], nullptr, s->tab + N, (void* const*)(s->tab + 3 * N), s->pitch[1],
                                    (int)s->lw[1], (int)s->lh[1], (int)N, inv_count, out_storage, st);
      });
      if (e != cudaSuccess) return cuda_err(ctx, e, "level-0 mask reduce");
    }
    // levels l >= 1 with enough tiles to fill the GPU: the blend of the level
    // and its mask REDUCE to l + 1 in one pass over every frame
    uint32_t lf = 1;
    for (; lf + 1 < s->L && lf < tail; ++lf) {
      const int64_t tiles = (int64_t)((s->lw[lf] + kTileW - 1) / kTileW) * ((s->lh[lf] + kTileH - 1) / kTileH);
      if (tiles < s->fuse_min_tiles) break;
      const void* const* lap = (const void* const*)(s->tab + (size_t)lf * 2 * N);
      const void* const* msk = (const void* const*)(s->tab + (size_t)lf * 2 * N + N);
      void* const* nxt = (void* const*)(s->tab + (size_t)(lf + 1) * 2 * N + N);
      const int out_storage = lf + 2 < s->L ? s->storage : FS_STORAGE_F32;
      e = timed(ctx, "level", [&] {
        return launch_blend_reduce(s->acc[lf], s->pitch[lf] * s->lh[lf], s->pitch[lf], (int)s->lw[lf], (int)s->lh[lf],
                                   s->sm[lf], lap, msk, nxt, s->pitch[lf + 1], (int)s->lw[lf + 1],
                                   (int)s->lh[lf + 1], (int)N, s->storage, out_storage, st);
      });
      if (e != cudaSuccess) return cuda_err(ctx, e, "level blend + mask reduce");
    }
    for (uint32_t l = lf; l + 1 < s->L && l < tail; ++l)
      if ((e = mask_reduce(l)) != cudaSuccess) return cuda_err(ctx, e, "mask reduce");
    // the blend of the other levels up to L-1 over every frame (top: Gaussian x mask)
    for (uint32_t l = lf; l < s->L && l < tail; ++l) {
      const void* const* lap = (const void* const*)(s->tab + (size_t)l * 2 * N);
      const void* const* msk = (const void* const*)(s->tab + (size_t)l * 2 * N + N);
      const int storage = l + 1 < s->L ? s->storage : FS_STORAGE_F32;
      e = timed(ctx, "level", [&] {
        return launch_blend(s->acc[l], s->pitch[l] * s->lh[l], s->pitch[l], (int)s->lw[l], (int)s->lh[l], lap, msk,
                            (int)N, storage, st);
      });
      if (e != cudaSuccess) return cuda_err(ctx, e, "level blend");
    }
    if (tail < s->L) {
      // levels tail .. L-1: masks, blends and their collapse in two launches
      BlendTailArgs b;
      std::memset(&b, 0, sizeof(b));
      b.first = (int32_t)tail;
      b.levels = (int32_t)s->L;
      b.frames = (int32_t)N;
      b.storage = s->storage;
      b.tab = (const void* const*)s->tab;
      b.sm_first = s->sm[tail];
      b.counter = s->tail_counter;
      for (uint32_t l = tail; l < s->L; ++l)
        b.lv[l - tail] = TailLevel{(int32_t)s->lw[l], (int32_t)s->lh[l], s->pitch[l], s->acc[l],
                                   s->pitch[l] * s->lh[l]};
      e = timed(ctx, "level", [&] { return launch_mask_tail(b, st); });
      if (e == cudaSuccess) e = timed(ctx, "level", [&] { return launch_blend_tail(b, st); });
      if (e != cudaSuccess) return cuda_err(ctx, e, "small-level tail");
      s->tail_folded = true;
    }
    return FS_OK;
  }
  std::vector<fs_stack::Frame> frames = s->frames;
  for (size_t begin = 0; begin < N; begin += s->K) {
    const size_t end = std::min(N, begin + s->K);
    if (s->mode == P2_RESIDENT || s->mode == P2_REFETCH) {
      for (size_t k = begin; k < end; ++k) {
        fs_stack::Frame& fr = frames[k];
        if (fr.resident) continue;
        // the frame was only staged for pass 1: fetch it again from the host
        // (the reference re-decodes, src/stack/pipeline.zig:561-597)
        if (!refetch) return set_err(ctx, FS_ERR_STATE, "frame not resident and no refetch callback");
        const void* hp = nullptr;
        size_t hs = 0;
        if (refetch(user, (uint32_t)k, &hp, &hs) != 0 || !hp)
          return set_err(ctx, FS_ERR_INVALID, "refetch callback failed");
        const size_t row_bytes = (size_t)s->d.src_width * s->d.channels * s->bps;
        if (hs < row_bytes) return set_err(ctx, FS_ERR_MISMATCH, "refetched row stride too small");
        uint8_t* buf = s->staging[(k - begin) % s->staging.size()];
        e = cudaMemcpy2DAsync(buf, (size_t)s->frame_pitch, hp, hs, row_bytes, s->d.src_height,
                              cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_err(ctx, e, "frame refetch upload");
        e = cudaStreamSynchronize(st);  // the callback's buffer may be reused after it returns again
        if (e != cudaSuccess) return cuda_err(ctx, e, "frame refetch upload");
        fr.px = buf;
        fr.pitch = s->frame_pitch;
      }
      rc = s->bps == 2 ? launch_remap16_batch(s, frames, begin, end, false, inv_count)
                       : launch_remap_weights_batch(s, frames, begin, end, false);
      if (rc != FS_OK) return rc;
      if (s->bps == 2 && s->L == 1) continue;  // blended with the planes (1 x 1 stack)
    }
    if (s->best) {
      // hybrid: the hardmask winners of this batch, from its pass-2 planes
      FramePlanes pl[kMaxBatch];
      for (size_t k = begin; k < end; ++k) pl[k - begin] = s->mode == P2_CACHE ? s->cache[k] : s->p2[k - begin];
      e = timed(ctx, "winners", [&] {
        return launch_winners(pl, (int)(end - begin), s->best, s->hard, begin == 0 ? 1 : 0, (int)s->W, (int)s->H,
                              s->pitch[0], st);
      });
      if (e != cudaSuccess) return cuda_err(ctx, e, "winners");
    }
    LevelArgs a;
    std::memset(&a, 0, sizeof(a));
    a.levels = (int32_t)s->L;
    a.K = (int32_t)(end - begin);
    a.inv_count = inv_count;
    a.norm = s->norm;
    for (size_t k = begin; k < end; ++k) {
      if (s->bps == 2) a.in[k - begin] = s->slot0[k - begin];  // level 0 of 16-bit frames: f32 planes
      else a.in0[k - begin] = s->mode == P2_CACHE ? s->cache[k] : s->p2[k - begin];
    }
    for (uint32_t l = 0; l + 1 < s->L || (s->L == 1 && l == 0); ++l) {
      a.level = (int32_t)l;
      a.wl = (int32_t)s->lw[l];
      a.hl = (int32_t)s->lh[l];
      a.pitch_l = s->pitch[l];
      a.exact_expand = std::max(s->lw[l], s->lh[l]) <= kExactExpandMaxDim ? 1 : 0;
      a.sm_l = s->sm[l];
      a.acc_l = s->acc[l];
      a.acc_plane_l = s->pitch[l] * s->lh[l];
      if (l + 1 < s->L) {
        a.wn = (int32_t)s->lw[l + 1];
        a.hn = (int32_t)s->lh[l + 1];
        a.pitch_n = s->pitch[l + 1];
        a.acc_n = s->acc[l + 1];
        a.acc_plane_n = s->pitch[l + 1] * s->lh[l + 1];
      } else {
        a.wn = a.hn = 1;
        a.pitch_n = 32;
      }
      for (size_t k = 0; k < (size_t)a.K; ++k) {
        if (l >= 1) a.in[k] = s->slot[k][l];
        if (l + 1 < s->L - 1) a.out[k] = s->slot[k][l + 1];
      }
      const bool fp = l >= 1 && l >= s->fp_level && s->contrib && a.K > 1;
      a.frame_parallel = fp ? 1 : 0;
      a.contrib = fp ? s->contrib : nullptr;
      a.contrib_top = fp ? s->contrib_top : nullptr;
      if (l == 0 && s->bps == 2) e = timed(ctx, "level0", [&] { return launch_level(a, FS_STORAGE_F32, st); });
      else if (l == 0) e = timed(ctx, "level0", [&] { return launch_level0(a, s->storage, st); });
      else e = timed(ctx, "level", [&] { return launch_level(a, s->storage, st); });
      if (e != cudaSuccess) return cuda_err(ctx, e, "level launch");
      if (fp) {
        // the frames' contributions into the accumulators, in frame order
        e = timed(ctx, "level", [&] {
          return launch_sum_contrib(a.acc_l, a.acc_plane_l, a.pitch_l, a.wl, a.hl, s->contrib, a.K, st);
        });
        if (e == cudaSuccess && l + 1 == s->L - 1)
          e = timed(ctx, "level", [&] {
            return launch_sum_contrib(a.acc_n, a.acc_plane_n, a.pitch_n, a.wn, a.hn, s->contrib_top, a.K, st);
          });
        if (e != cudaSuccess) return cuda_err(ctx, e, "contribution sum");
      }
      if (s->L == 1) break;
    }
  }
  return FS_OK;
}

// Collapse kernels of the accumulator pyramid into the quantised output
// out_dev, with the collapsed base into `base` when given, from level `top`
// down (levels above it already added into it).
static int collapse_kernels(fs_stack* s, float* base, uint32_t top) {
  fs_ctx* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  if (s->L == 1) {
    e = timed(ctx, "collapse", [&] {
      return launch_quantize(s->acc[0], s->pitch[0] * s->lh[0], s->pitch[0], (int)s->W, (int)s->H, s->out_dev,
                             (int64_t)s->W * 3 * s->bps, base, s->base_pitch, s->bps == 2, st);
    });
    if (e != cudaSuccess) return cuda_err(ctx, e, "quantise");
  }
  for (uint32_t l = std::min(top, s->L - 1); l >= 1 && s->L > 1; --l) {
    CollapseArgs c;
    std::memset(&c, 0, sizeof(c));
    c.wp = (int32_t)s->lw[l - 1];
    c.hp = (int32_t)s->lh[l - 1];
    c.wc = (int32_t)s->lw[l];
    c.hc = (int32_t)s->lh[l];
    c.pitch_p = s->pitch[l - 1];
    c.pitch_c = s->pitch[l];
    c.exact_expand = std::max(s->lw[l - 1], s->lh[l - 1]) <= kExactExpandMaxDim ? 1 : 0;
    c.acc_p = s->acc[l - 1];
    c.plane_p = s->pitch[l - 1] * s->lh[l - 1];
    c.acc_c = s->acc[l];
    c.plane_c = s->pitch[l] * s->lh[l];
    c.out = l == 1 ? s->out_dev : nullptr;
    c.out_pitch = (int64_t)s->W * 3 * s->bps;
    c.out16 = s->bps == 2 ? 1 : 0;
    c.base = l == 1 ? base : nullptr;
    c.base_pitch = s->base_pitch;
    e = timed(ctx, "collapse", [&] { return launch_collapse(c, st); });
    if (e != cudaSuccess) return cuda_err(ctx, e, "collapse");
  }
  return FS_OK;
}

// hybrid-pyramid-contrast: the plain Laplacian pyramids of the soft image
// (the pyramid-contrast output in out_dev) and of the hard image (the
// winners' colours), merged into the accumulator pyramid
// (mergeHybridImages, src/fuse/pyramid.zig:271-301; hard levels from
// hybrid_hard_level_start = 2, hybrid_hard_level_count = 4, :9-10).
static int hybrid_merge(fs_stack* s) {
  fs_ctx* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  std::vector<float*> gs(s->L), gh(s->L);
  for (uint32_t l = 0; l < s->L; ++l) {
    void* p;
    const size_t bytes = (size_t)s->pitch[l] * s->lh[l] * 12;
    int rc = stack_alloc(s, bytes, &p);
    if (rc == FS_OK) {
      gs[l] = (float*)p;
      rc = stack_alloc(s, bytes, &p);
    }
    if (rc != FS_OK) return rc;
    gh[l] = (float*)p;
  }
  auto plane = [&](uint32_t l) { return s->pitch[l] * s->lh[l]; };
  e = timed(ctx, "hybrid", [&] {
    return launch_rgb_to_planes(s->out_dev, (int64_t)s->W * 3, 3, gs[0], plane(0), s->pitch[0], (int)s->W, (int)s->H,
                                st);
  });
  if (e == cudaSuccess)
    e = timed(ctx, "hybrid", [&] {
      return launch_rgb_to_planes((const uint8_t*)s->hard, s->pitch[0] * 4, 4, gh[0], plane(0), s->pitch[0],
                                  (int)s->W, (int)s->H, st);
    });
  for (uint32_t l = 0; e == cudaSuccess && l + 1 < s->L; ++l) {
    for (std::vector<float*>* g : {&gs, &gh}) {
      e = timed(ctx, "hybrid", [&] {
        return launch_reduce_plain((*g)[l], plane(l), s->pitch[l], (int)s->lw[l], (int)s->lh[l], (*g)[l + 1],
                                   plane(l + 1), s->pitch[l + 1], (int)s->lw[l + 1], (int)s->lh[l + 1], st);
      });
      if (e != cudaSuccess) break;
    }
  }
  const uint32_t hs = std::min<uint32_t>(2, s->L), he = std::min<uint32_t>(hs + 4, s->L);
  for (uint32_t l = 0; e == cudaSuccess && l + 1 < s->L; ++l) {
    MergeArgs m;
    std::memset(&m, 0, sizeof(m));
    m.wp = (int32_t)s->lw[l];
    m.hp = (int32_t)s->lh[l];
    m.wc = (int32_t)s->lw[l + 1];
    m.hc = (int32_t)s->lh[l + 1];
    m.pitch_p = s->pitch[l];
    m.pitch_c = s->pitch[l + 1];
    m.plane_p = plane(l);
    m.plane_c = plane(l + 1);
    m.exact_expand = std::max(s->lw[l], s->lh[l]) <= kExactExpandMaxDim ? 1 : 0;
    m.mixed = l >= hs && l < he ? 1 : 0;
    m.mix = s->hybrid_mix;
    m.soft_p = gs[l];
    m.hard_p = gh[l];
    m.soft_c = gs[l + 1];
    m.hard_c = gh[l + 1];
    m.acc = s->acc[l];
    e = timed(ctx, "hybrid", [&] { return launch_merge_level(m, st); });
  }
  if (e == cudaSuccess) {
    const uint32_t t = s->L - 1;
    e = timed(ctx, "hybrid", [&] {
      return launch_merge_top(gs[t], gh[t], s->acc[t], plane(t), s->pitch[t], (int)s->lw[t], (int)s->lh[t],
                              t >= hs && t < he ? 1 : 0, s->hybrid_mix, st);
    });
  }
  if (e != cudaSuccess) return cuda_err(ctx, e, "hybrid merge");
  return FS_OK;
}

// Collapse of the accumulator pyramid and the quantised output
// (src/fuse/pyramid.zig:223-269); the hybrid method collapses twice (the
// soft image, then the merged pyramid).
static int collapse_impl(fs_stack* s, void* out, size_t out_stride, bool device_out, bool wait) {
  fs_ctx* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  int rc;
  if (s->best) {
    // the soft image, then the merged pyramid (written whole by the merge)
    if ((rc = collapse_kernels(s, nullptr, s->tail_folded ? s->tail : s->L - 1)) != FS_OK) return rc;
    if ((rc = hybrid_merge(s)) != FS_OK) return rc;
    s->tail_folded = false;
  }
  if ((rc = collapse_kernels(s, s->base_out, s->tail_folded ? s->tail : s->L - 1)) != FS_OK) return rc;
  const cudaMemcpyKind kind = device_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t row = (size_t)s->W * 3 * s->bps;
  if (out_stride == row)
    e = cudaMemcpyAsync(out, s->out_dev, row * s->H, kind, st);
  else
    e = cudaMemcpy2DAsync(out, out_stride, s->out_dev, row, row, s->H, kind, st);
  if (e != cudaSuccess) return cuda_err(ctx, e, "output copy");
  if (wait) {
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_err(ctx, e, "fusion");
  }
  return FS_OK;
}

int fs_stack_set_method(fs_stack* s, int method, float hybrid_sharpness) {
  if (!s) return FS_ERR_INVALID;
  if (!s->ctx) return FS_ERR_STATE;
  if (method != FS_METHOD_PYRAMID_CONTRAST && method != FS_METHOD_HYBRID_PYRAMID_CONTRAST)
    return set_err(s->ctx, FS_ERR_INVALID, "unknown fusion method");
  if (!(hybrid_sharpness >= 0.0f && hybrid_sharpness <= 1.0f))  // parseSharpness, src/fuse/config.zig:269-273
    return set_err(s->ctx, FS_ERR_INVALID, "hybrid sharpness must be in [0, 1]");
  if (!s->frames.empty() || s->finished) return set_err(s->ctx, FS_ERR_STATE, "method set after the first frame");
  if (s->frame_total) return set_err(s->ctx, FS_ERR_UNSUPPORTED, "the hybrid method does not run frame-sharded");
  s->method = method;
  s->hybrid_mix = hybrid_sharpness;
  if (method == FS_METHOD_HYBRID_PYRAMID_CONTRAST && !s->best) {
    if (s->bps != 1) return set_err(s->ctx, FS_ERR_UNSUPPORTED, "the hybrid method takes 8-bit samples");
    cudaSetDevice(s->ctx->device);
    const size_t n0 = (size_t)s->pitch[0] * s->H;
    void* p;
    int rc = stack_alloc(s, n0 * 4, &p);
    if (rc != FS_OK) return rc;
    s->best = (float*)p;
    if ((rc = stack_alloc(s, n0 * 4, &p)) != FS_OK) return rc;
    s->hard = (uint32_t*)p;
  }
  return FS_OK;
}

int fs_stack_pass2_mode(const fs_stack* s) { return s ? (int)s->mode : -1; }

int fs_stack_mode_bytes(const fs_stack_desc* desc, int pass2_mode, int host_frames, uint64_t* bytes) {
  if (!desc || !bytes || pass2_mode < 0 || pass2_mode > P2_FUSED) return FS_ERR_INVALID;
  int code = FS_OK;
  if (check_desc(*desc, &code)) return code;
  const StackPlan plan = plan_stack(*desc);
  if (pass2_mode >= P2_LAPS && plan.laps_frame == 0) return FS_ERR_UNSUPPORTED;
  if (desc->sample_bits == 16 && (pass2_mode == P2_CACHE || pass2_mode >= P2_LAPS)) return FS_ERR_UNSUPPORTED;
  *bytes = plan_bytes(plan, desc->frame_count, (Pass2Mode)pass2_mode, host_frames != 0);
  return FS_OK;
}

int fs_stack_footprint(const fs_stack_desc* desc, uint64_t available_bytes, int host_frames, uint64_t* bytes,
                       int* mode) {
  if (!desc || !bytes) return FS_ERR_INVALID;
  int code = FS_OK;
  if (check_desc(*desc, &code)) return code;
  const StackPlan plan = plan_stack(*desc);
  const Pass2Mode m = choose_mode(plan, desc->frame_count, available_bytes, host_frames != 0, desc->sample_bits == 16);
  *bytes = plan_bytes(plan, desc->frame_count, m, host_frames != 0);
  if (mode) *mode = (int)m;
  return *bytes <= available_bytes ? FS_OK : FS_ERR_BUDGET;
}

// ------------------------------------------------ phases (frame-sharded stacks)
static int phase_check(fs_stack* s, int want) {
  if (!s) return FS_ERR_INVALID;
  if (!s->ctx) return FS_ERR_STATE;
  if (s->finished) return set_err(s->ctx, FS_ERR_STATE, "stack already finished");
  if (s->frames.size() != s->d.frame_count) return set_err(s->ctx, FS_ERR_STATE, "fewer frames added than frame_count");
  if (s->phase != want) return set_err(s->ctx, FS_ERR_STATE, "stack phase out of order");
  cudaSetDevice(s->ctx->device);
  return FS_OK;
}

int fs_stack_set_frame_total(fs_stack* s, uint32_t frame_total) {
  if (!s) return FS_ERR_INVALID;
  if (!s->ctx) return FS_ERR_STATE;
  if (frame_total < s->d.frame_count) return set_err(s->ctx, FS_ERR_INVALID, "total below this stack's frames");
  if (s->best) return set_err(s->ctx, FS_ERR_UNSUPPORTED, "the hybrid method does not run frame-sharded");
  s->frame_total = frame_total;
  return FS_OK;
}

int fs_stack_end_pass1(fs_stack* s) {
  int rc = phase_check(s, 0);
  if (rc != FS_OK) return rc;
  if ((rc = run_pending_pass1(s, true)) != FS_OK) return rc;
  cudaError_t e = cudaStreamSynchronize(s->ctx->stream);
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "pass 1");
  s->phase = 1;
  return FS_OK;
}

int fs_stack_blend(fs_stack* s, fs_frame_fetch_cb refetch, void* user) {
  int rc = phase_check(s, 1);
  if (rc != FS_OK) return rc;
  if ((rc = pass2_impl(s, refetch, user, false)) != FS_OK) return rc;
  cudaError_t e = cudaStreamSynchronize(s->ctx->stream);
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "pass 2");
  s->phase = 2;
  return FS_OK;
}

int fs_stack_collapse(fs_stack* s, void* out_pixels, size_t out_stride, int device_out) {
  int rc = phase_check(s, 2);
  if (rc != FS_OK) return rc;
  if (!out_pixels) return FS_ERR_INVALID;
  if (out_stride < (size_t)s->W * 3 * s->bps) return set_err(s->ctx, FS_ERR_INVALID, "output stride too small");
  if ((rc = collapse_impl(s, out_pixels, out_stride, device_out != 0, true)) != FS_OK) return rc;
  s->finished = true;
  return FS_OK;
}

int fs_stack_buffer(fs_stack* s, int which, uint32_t level, void** ptr, uint64_t* bytes, int64_t* pitch,
                    uint32_t* width, uint32_t* height) {
  if (!s || !ptr || !bytes) return FS_ERR_INVALID;
  if (!s->ctx) return FS_ERR_STATE;
  if (level >= s->L || (which != FS_BUFFER_ACCUMULATOR && level != 0))
    return set_err(s->ctx, FS_ERR_INVALID, "no such buffer");
  const size_t plane = (size_t)s->pitch[level] * s->lh[level];
  switch (which) {
    case FS_BUFFER_WEIGHT_SUM: *ptr = s->norm; *bytes = plane * 4; break;
    case FS_BUFFER_UNION: *ptr = s->uni; *bytes = plane; break;
    case FS_BUFFER_ACCUMULATOR: *ptr = s->acc[level]; *bytes = plane * 12; break;
    case FS_BUFFER_HARD:
      if (!s->hard) return set_err(s->ctx, FS_ERR_INVALID, "no hard image (pyramid-contrast stack)");
      *ptr = s->hard;
      *bytes = plane * 4;
      break;
    default: return set_err(s->ctx, FS_ERR_INVALID, "no such buffer");
  }
  if (pitch) *pitch = s->pitch[level];
  if (width) *width = s->lw[level];
  if (height) *height = s->lh[level];
  return FS_OK;
}

int fs_stack_finish(fs_stack* stack, fs_frame_fetch_cb refetch, void* user, void* out_pixels, size_t out_stride) {
  return finish_impl(stack, refetch, user, out_pixels, out_stride, false);
}

int fs_stack_finish_device(fs_stack* stack, fs_frame_fetch_cb refetch, void* user, void* dev_out, size_t out_stride) {
  return finish_impl(stack, refetch, user, dev_out, out_stride, true);
}

int fs_stack_finish_async(fs_stack* stack, fs_frame_fetch_cb refetch, void* user, void* out_pixels,
                          size_t out_stride) {
  return finish_impl(stack, refetch, user, out_pixels, out_stride, false, false, true);
}

int fs_stack_wait(fs_stack* s) {
  if (!s) return FS_ERR_INVALID;
  if (!s->ctx) return FS_ERR_STATE;
  if (!s->finished) return set_err(s->ctx, FS_ERR_STATE, "stack not finished");
  if (!s->done) return FS_OK;  // finished synchronously
  cudaSetDevice(s->ctx->device);
  const cudaError_t e = cudaEventSynchronize(s->done);
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "fusion");
  return FS_OK;
}

int fs_stack_set_base_output(fs_stack* s, float* dev_base, size_t row_stride_elems) {
  if (!s) return FS_ERR_INVALID;
  if (!s->ctx) return FS_ERR_STATE;
  if (dev_base && row_stride_elems < (size_t)s->W * 3) return set_err(s->ctx, FS_ERR_INVALID, "base stride too small");
  s->base_out = dev_base;
  s->base_pitch = (int64_t)row_stride_elems;
  return FS_OK;
}

int fs_stack_output_size(const fs_stack* s, uint32_t* width, uint32_t* height) {
  if (!s) return FS_ERR_INVALID;
  if (width) *width = s->W;
  if (height) *height = s->H;
  return FS_OK;
}

int fs_stack_destroy(fs_stack* s) {
  if (!s) return FS_ERR_INVALID;
  if (fs_ctx* ctx = s->ctx) {
    cudaSetDevice(ctx->device);
    cudaStream_t free_on = ctx->stream;
    if (s->done) {
      // finished asynchronously: its last work is the output copy, so once
      // that is done nothing of it is in flight; its memory is freed on the
      // idle stream, where the frees complete at once and the pool can hand
      // it to the next stacks (the later stacks' work queued on the context's
      // streams need not drain first)
      cudaEventSynchronize(s->done);
      free_on = ctx->idle;
    } else {
      cudaStreamSynchronize(ctx->stream);
      cudaStreamSynchronize(ctx->copy);
    }
    for (auto& a : s->allocs) dev_free(ctx, a.p, a.bytes, free_on);
    s->allocs.clear();
    ctx->stacks.erase(s);
    detach_stack(s);
  }
  delete s;
  return FS_OK;
}

int fs_fuse_stack(fs_ctx* ctx, const fs_stack_desc* desc, const void* const* frames, const size_t* row_strides,
                  const fs_pose* poses, void* out_pixels, size_t out_stride) {
  if (!ctx || !desc || !frames || !row_strides || !out_pixels) return set_err(ctx, FS_ERR_INVALID, "null argument");
  fs_stack* s = nullptr;
  int rc = fs_stack_begin(ctx, desc, &s);
  if (rc != FS_OK) return rc;
  for (uint32_t k = 0; k < desc->frame_count && rc == FS_OK; ++k)
    rc = fs_stack_add_frame(s, frames[k], row_strides[k], poses ? &poses[k] : nullptr);
  if (rc == FS_OK) rc = fs_stack_finish(s, nullptr, nullptr, out_pixels, out_stride);
  fs_stack_destroy(s);
  return rc;
}

// ---------------------------------------------------------------- synthetic
int fs_synth_pose(uint64_t seed, int scene, uint32_t width, uint32_t height, uint32_t frame, uint32_t frame_count,
                  fs_pose* pose_out) {
  if (!pose_out) return FS_ERR_INVALID;
  synth_pose(seed, scene, width, height, frame, frame_count, pose_out);
  return FS_OK;
}

int fs_synth_frame_device(fs_ctx* ctx, uint64_t seed, int scene, uint32_t width, uint32_t height, uint32_t frame,
                          uint32_t frame_count, void* dev_out, size_t out_stride, fs_pose* pose_out) {
  if (!ctx || !dev_out) return set_err(ctx, FS_ERR_INVALID, "null argument");
  if (out_stride < (size_t)width * 3) return set_err(ctx, FS_ERR_INVALID, "stride too small");
  cudaSetDevice(ctx->device);
  const char* why = nullptr;
  int rc = synth_render(seed, scene, width, height, frame, frame_count, dev_out, out_stride, pose_out, ctx->stream,
                        &why);
  if (rc != FS_OK) return set_err(ctx, rc, why ? why : "synthetic render failed");
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_err(ctx, e, "synthetic render");
  return FS_OK;
}

}  // extern "C"

// ================================================================= batches
// Batched form: many independent stacks over device-resident frames, spread
// over `lanes` contexts (streams) and run as one CUDA graph: the first
// fs_batch_run executes the work directly (and configures the kernels), the
// second captures the same launch sequence, every later run replays it with
// one graph launch.  The stacks of a lane run one after another on its
// stream, so they share one device arena, sized for the lane's largest
// stack: a batch holds (lanes x its largest stacks) bytes instead of the sum
// over all its stacks, which lets every stack take the split-pyramid modes.
// Every stack's state is re-initialised by the kernels of the run itself
// (pass 1 writes the weight sum, union and per-frame planes of the first
// batch, pass 2 clears or writes the accumulators whole), so a replay
// recomputes every stack from the frames at the same device addresses; only
// the split-pyramid frame tables, written once at create, live outside the
// arenas.
struct fs_batch {
  fs_ctx* parent = nullptr;
  std::vector<fs_ctx*> lanes;
  struct Item {
    fs_stack* stack = nullptr;
    int lane = 0;
    std::vector<const void*> frames;
    size_t stride = 0;
    std::vector<fs_pose> poses;
    void* out = nullptr;
    size_t out_stride = 0;
  };
  std::vector<Item> items;
  std::vector<void*> arenas;         // per lane
  std::vector<uint64_t> arena_bytes;
  std::vector<cudaEvent_t> join;
  std::vector<int> planned;  // pass-2 mode of each stack
  uint64_t charged = 0;      // device bytes counted against the parent's budget
  cudaEvent_t fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int runs = 0;
};

namespace {

int batch_enqueue(fs_batch* b) {
  // lane by lane, each lane's stacks in order (they share its arena)
  for (size_t l = 0; l < b->lanes.size(); ++l) {
    for (auto& it : b->items) {
      if (it.lane != (int)l) continue;
      fs_stack* s = it.stack;
      s->frames.clear();
      s->pass1_done = 0;
      s->finished = false;
      s->phase = 0;
      for (size_t k = 0; k < it.frames.size(); ++k) {
        const fs_pose* pose = s->aligned ? nullptr : &it.poses[k];
        int rc = add_frame_impl(s, it.frames[k], it.stride, pose, true);
        if (rc != FS_OK) return rc;
      }
      int rc = finish_impl(s, nullptr, nullptr, it.out, it.out_stride, true, false);
      if (rc != FS_OK) return rc;
    }
  }
  return FS_OK;
}

// Fork every lane from the parent stream, enqueue, join back.
int batch_enqueue_forked(fs_batch* b) {
  fs_ctx* P = b->parent;
  cudaEventRecord(b->fork, P->stream);
  for (fs_ctx* l : b->lanes) cudaStreamWaitEvent(l->stream, b->fork, 0);
  int rc = batch_enqueue(b);
  for (size_t i = 0; i < b->lanes.size(); ++i) {
    cudaEventRecord(b->join[i], b->lanes[i]->stream);
    cudaStreamWaitEvent(P->stream, b->join[i], 0);
  }
  return rc;
}

// Arena bytes of one stack in mode m: its plan plus the 256-byte rounding of
// every piece (at most this many pieces: fixed state, level slots, batch
// slots, per-frame planes).
uint64_t arena_need(const StackPlan& p, uint32_t frames, Pass2Mode m) {
  const uint64_t pieces = 9 + 3ull * p.L + (uint64_t)p.K * (p.L + 1) + frames;
  return plan_bytes(p, frames, m, false) + pieces * kArenaAlign;
}

// The split-pyramid frame table of a stack and the tail counter after it
// (allocated from the lane's pool).
uint64_t table_bytes(const StackPlan& p, uint32_t frames, Pass2Mode m) {
  return (m == P2_LAPS || m == P2_FUSED) ? 2ull * p.L * frames * sizeof(float*) + 16 : 0;
}

// The stack's mode when the batch asks for `want`: the split-pyramid modes
// need three levels or more (smaller stacks cache their planes).
Pass2Mode stack_mode(const StackPlan& p, Pass2Mode want) {
  if (want == P2_LAPS && !p.laps_frame) return P2_CACHE;
  if (want == P2_FUSED && !p.fused_frame) return P2_CACHE;
  return want;
}

}  // namespace

int fs_batch_create(fs_ctx* ctx, uint32_t n, const fs_stack_desc* descs, const void* const* const* frames,
                    const size_t* row_strides, const fs_pose* const* poses, void* const* dev_out,
                    const size_t* out_strides, uint32_t lanes, int pass2_mode, fs_batch** out) {
  if (!ctx || !descs || !frames || !row_strides || !dev_out || !out_strides || !out || n == 0)
    return set_err(ctx, FS_ERR_INVALID, "null argument");
  if (pass2_mode < -1 || pass2_mode > P2_FUSED || pass2_mode == P2_REFETCH)
    return set_err(ctx, FS_ERR_INVALID, "pass2_mode must be -1, 0 (cache), 1 (resident), 3 (laps) or 4 (fused)");
  *out = nullptr;
  lanes = std::max(1u, std::min(lanes, n));
  cudaSetDevice(ctx->device);
  fs_batch* b = new fs_batch();
  b->parent = ctx;
  auto fail = [&](int rc) {
    fs_batch_destroy(b);
    return rc;
  };
  std::vector<StackPlan> plans;
  std::vector<double> work(n);
  for (uint32_t i = 0; i < n; ++i) {
    int code = FS_OK;
    if (const char* why = check_desc(descs[i], &code)) return fail(set_err(ctx, code, why));
    if (descs[i].sample_bits != 8) return fail(set_err(ctx, FS_ERR_UNSUPPORTED, "batches take 8-bit stacks"));
    if (!frames[i]) return fail(set_err(ctx, FS_ERR_INVALID, "null frame list"));
    if (!descs[i].input_is_aligned && !poses) return fail(set_err(ctx, FS_ERR_INVALID, "poses required"));
    plans.push_back(plan_stack(descs[i]));
    work[i] = (double)descs[i].frame_count * plans[i].W * plans[i].H;
  }
  // lanes: largest stack first to the least-loaded lane (frame-pixels)
  std::vector<uint32_t> order(n);
  for (uint32_t i = 0; i < n; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t c) { return work[a] > work[c]; });
  std::vector<double> load(lanes, 0.0);
  b->items.resize(n);
  for (uint32_t i : order) {
    const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[l] += work[i];
    b->items[i].lane = l;
  }
  // mode: the one asked for, or the fastest whose lane arenas fit the budget
  // (split pyramid, then fused, then cached planes, then frames kept)
  const uint64_t left = ctx->budget > ctx->held ? ctx->budget - ctx->held : 0;
  std::vector<uint64_t> arena(lanes), tables(lanes);
  auto size_lanes = [&](Pass2Mode want) {
    std::fill(arena.begin(), arena.end(), 0);
    std::fill(tables.begin(), tables.end(), 0);
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i) {
      const Pass2Mode m = stack_mode(plans[i], want);
      const int l = b->items[i].lane;
      arena[l] = std::max(arena[l], arena_need(plans[i], descs[i].frame_count, m));
      tables[l] += table_bytes(plans[i], descs[i].frame_count, m) + kArenaAlign;
    }
    for (uint32_t l = 0; l < lanes; ++l) total += arena[l] + tables[l];
    return total;
  };
  Pass2Mode want = P2_CACHE;
  uint64_t total = 0;
  if (pass2_mode >= 0) {
    want = (Pass2Mode)pass2_mode;
    total = size_lanes(want);
  } else {
    for (Pass2Mode m : {P2_LAPS, P2_FUSED, P2_CACHE, P2_RESIDENT}) {
      want = m;
      if ((total = size_lanes(m)) <= left) break;
    }
  }
  if (total > left)
    return fail(set_err(ctx, FS_ERR_BUDGET, "batch needs " + std::to_string(total) + " device bytes, budget leaves " +
                                                std::to_string(left)));
  for (uint32_t i = 0; i < n; ++i) b->planned.push_back((int)stack_mode(plans[i], want));
  for (uint32_t l = 0; l < lanes; ++l) {
    fs_ctx* c = nullptr;
    int rc = fs_create(ctx->device, std::max<uint64_t>(arena[l] + tables[l], 1), &c);
    if (rc != FS_OK) return fail(rc);
    c->fuse_min_tiles = ctx->fuse_min_tiles;  // the lanes' stacks take the parent's level schedule
    c->tail_side = ctx->tail_side;
    b->lanes.push_back(c);
    cudaEvent_t ev;
    cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    b->join.push_back(ev);
    void* p = nullptr;
    if (arena[l] && (rc = dev_alloc(c, arena[l], &p)) != FS_OK)
      return fail(set_err(ctx, rc, std::string("lane arena: ") + fs_last_error(c)));
    b->arenas.push_back(p);
    b->arena_bytes.push_back(arena[l]);
  }
  cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (uint32_t i = 0; i < n; ++i) {
    auto& it = b->items[i];
    fs_ctx* lc = b->lanes[it.lane];
    int rc = begin_impl(lc, &descs[i], &it.stack, b->planned[i], (uint8_t*)b->arenas[it.lane],
                        b->arena_bytes[it.lane]);
    if (rc != FS_OK) return fail(set_err(ctx, rc, std::string("stack begin: ") + fs_last_error(lc)));
    it.frames.assign(frames[i], frames[i] + descs[i].frame_count);
    it.stride = row_strides[i];
    if (!descs[i].input_is_aligned) it.poses.assign(poses[i], poses[i] + descs[i].frame_count);
    it.out = dev_out[i];
    it.out_stride = out_strides[i];
    if (!it.out || it.out_stride < (size_t)it.stack->W * 3) return fail(set_err(ctx, FS_ERR_INVALID, "bad output"));
  }
  // the frame tables' uploads are done before the lanes' streams read them
  for (fs_ctx* c : b->lanes) cudaStreamSynchronize(c->stream);
  ctx->held += total;  // the lanes' memory counts against the parent's budget
  b->charged = total;
  b->runs = 0;
  *out = b;
  return FS_OK;
}

int fs_batch_run(fs_batch* b) {
  if (!b) return FS_ERR_INVALID;
  fs_ctx* P = b->parent;
  cudaSetDevice(P->device);
  cudaError_t e;
  if (b->runs == 0) {
    int rc = batch_enqueue_forked(b);  // direct execution, configures every kernel
    if (rc != FS_OK) return rc;
  } else {
    if (!b->exec) {
      e = cudaStreamBeginCapture(P->stream, cudaStreamCaptureModeRelaxed);
      if (e != cudaSuccess) return cuda_err(P, e, "begin capture");
      int rc = batch_enqueue_forked(b);
      cudaGraph_t g = nullptr;
      e = cudaStreamEndCapture(P->stream, &g);
      if (rc != FS_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (e != cudaSuccess) return cuda_err(P, e, "end capture");
      b->graph = g;
      e = cudaGraphInstantiate(&b->exec, g, 0);
      if (e != cudaSuccess) return cuda_err(P, e, "graph instantiate");
    }
    e = cudaGraphLaunch(b->exec, P->stream);
    if (e != cudaSuccess) return cuda_err(P, e, "graph launch");
  }
  e = cudaStreamSynchronize(P->stream);
  if (e != cudaSuccess) return cuda_err(P, e, "batch");
  ++b->runs;
  return FS_OK;
}

int fs_batch_stack_count(const fs_batch* b) { return b ? (int)b->items.size() : -1; }

int fs_batch_pass2_mode(const fs_batch* b, uint32_t i) {
  return (b && i < b->items.size()) ? (int)b->items[i].stack->mode : -1;
}

int fs_batch_uses_graph(const fs_batch* b) { return (b && b->exec) ? 1 : 0; }

int fs_batch_destroy(fs_batch* b) {
  if (!b) return FS_ERR_INVALID;
  if (b->parent) cudaStreamSynchronize(b->parent->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto& it : b->items)
    if (it.stack) fs_stack_destroy(it.stack);
  for (size_t l = 0; l < b->arenas.size(); ++l) dev_free(b->lanes[l], b->arenas[l], b->arena_bytes[l]);
  for (fs_ctx* c : b->lanes) fs_destroy(c);
  for (cudaEvent_t ev : b->join) cudaEventDestroy(ev);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->parent) b->parent->held -= std::min(b->parent->held, b->charged);
  delete b;
  return FS_OK;
}
