// Context-free fusion of a small pre-aligned stack whose intermediate planes
// live in one file-scope device array, so the call allocates nothing.
//
// Who needs it: a caller that must not allocate device memory while it runs.
// cudaFree waits for the whole device and cudaMalloc can wait behind other
// streams, so a host that interleaves this fusion with its own kernels (an
// interactive preview loop, a server that reserved its HBM when it started
// and accounts for every byte after that) cannot pay for either, and a host
// that lends the plugin only buffers it owns does not want the plugin's
// footprint to grow per call.  Such a caller passes device frames, a device
// output and its own stream; the planes of the pyramid come from the array
// below, whose size is fixed when the module loads.
//
// The array is shared by every call in the process on a given device.  Two
// calls in flight at the same time (on different streams, or from different
// host threads) overwrite each other's planes: callers order them (same
// stream, or an event between them).  Only the per-level accumulators must
// start at zero; each call clears them on its own stream before use.  The
// weight sum and the union are written (not added) by the first batch, and
// every other plane is written before it is read.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

#include "../../include/focuscuda.h"
#include "fusion_kernels.cuh"

namespace fs {
namespace {

// 40 MiB: 8 aligned frames of 512 x 512, or fewer / smaller frames, fit.
constexpr size_t kStaticScratchBytes = 40ull << 20;

__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

void put_err(char* err, size_t err_len, const char* fmt, ...) __attribute__((format(printf, 3, 4)));
void put_err(char* err, size_t err_len, const char* fmt, ...) {
  if (!err || err_len == 0) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(err, err_len, fmt, ap);
  va_end(ap);
}

// Device address of the scratch array in the current device's context.  The
// first call on a device loads the module there (the set-up step: make it
// before any stream capture); later calls are a table lookup in the CUDA
// runtime.  The address is looked up on every call and never cached, so a
// device that was reset, or another context made current, gets the address
// of its own copy of the array.
int scratch_on_current_device(unsigned char** out, char* err, size_t err_len) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    put_err(err, err_len, "cudaGetDevice: %s", cudaGetErrorString(e));
    return FS_ERR_NO_DEVICE;
  }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_static_scratch);
  if (e != cudaSuccess || !p) {
    put_err(err, err_len, "cudaGetSymbolAddress(static scratch) on device %d: %s", dev,
            e != cudaSuccess ? cudaGetErrorString(e) : "null address");
    return e == cudaErrorNoKernelImageForDevice || e == cudaErrorInvalidDevice ? FS_ERR_NO_DEVICE : FS_ERR_CUDA;
  }
  *out = (unsigned char*)p;
  return FS_OK;
}

// Offsets of every plane of a stack of `count` frames of w x h in the
// scratch array (level pitches rounded to 32 elements, each region aligned
// to 256 bytes), the same planes a context-backed stack allocates.
struct StaticLayout {
  uint32_t L = 0;
  uint32_t lw[32], lh[32];
  int64_t pitch[32];
  size_t norm, uni, sm[32], acc[32], planes[kMaxBatch], slot[kMaxBatch][32];
  size_t bytes = 0;
};

size_t take(size_t* cursor, size_t bytes) {
  const size_t at = *cursor;
  *cursor += (bytes + 255) & ~(size_t)255;
  return at;
}

void plan_layout(uint32_t w, uint32_t h, uint32_t count, StaticLayout* lay) {
  lay->L = level_count(w, h);
  for (uint32_t l = 0; l < lay->L; ++l) {
    lay->lw[l] = w;
    lay->lh[l] = h;
    lay->pitch[l] = ((int64_t)w + 31) / 32 * 32;
    w = next_level_size(w);
    h = next_level_size(h);
  }
  size_t c = 0;
  const size_t n0 = (size_t)lay->pitch[0] * lay->lh[0];
  lay->norm = take(&c, n0 * 4);
  lay->uni = take(&c, n0);
  lay->sm[0] = lay->uni;
  for (uint32_t l = 1; l < lay->L; ++l) lay->sm[l] = take(&c, (size_t)lay->pitch[l] * lay->lh[l]);
  for (uint32_t l = 0; l < lay->L; ++l) lay->acc[l] = take(&c, (size_t)lay->pitch[l] * lay->lh[l] * 12);
  for (uint32_t k = 0; k < count; ++k) {
    lay->planes[k] = take(&c, n0 * 8);
    for (uint32_t l = 1; l + 1 < lay->L; ++l) lay->slot[k][l] = take(&c, (size_t)lay->pitch[l] * lay->lh[l] * 17);
  }
  lay->bytes = c;
}

}  // namespace
}  // namespace fs

using namespace fs;

extern "C" int fs_fuse_aligned_device_static(const void* const* dev_frames, const size_t* row_strides,
                                             uint32_t frame_count, uint32_t width, uint32_t height,
                                             uint32_t channels, uint32_t contrast_window, void* dev_out,
                                             size_t out_stride, void* stream, char* err, size_t err_len) {
  if (err && err_len) err[0] = '\0';
  if (!dev_frames || !row_strides || !dev_out) {
    put_err(err, err_len, "null argument");
    return FS_ERR_INVALID;
  }
  if (frame_count == 0 || width == 0 || height == 0) {
    put_err(err, err_len, "empty stack");
    return FS_ERR_INVALID;
  }
  if (channels != 3 && channels != 4) {
    put_err(err, err_len, "channels must be 3 (RGB) or 4 (RGBA)");
    return FS_ERR_INVALID;
  }
  if (contrast_window < 3 || (contrast_window & 1) == 0) {
    put_err(err, err_len, "contrast window must be odd and >= 3");
    return FS_ERR_INVALID;
  }
  if (contrast_window > 2 * kMaxBorder + 1) {
    put_err(err, err_len, "contrast window larger than 15");
    return FS_ERR_UNSUPPORTED;
  }
  if (frame_count > (uint32_t)kMaxBatch) {
    put_err(err, err_len, "%u frames: the static-scratch fusion takes at most %d frames (one batch)", frame_count,
            kMaxBatch);
    return FS_ERR_UNSUPPORTED;
  }
  if (width > 8192 || height > 8192) {
    put_err(err, err_len, "%ux%u frames exceed the static scratch (40 MiB, e.g. 8 frames of 512x512)", width,
            height);
    return FS_ERR_UNSUPPORTED;
  }
  if (out_stride < (size_t)width * 3) {
    put_err(err, err_len, "output stride too small");
    return FS_ERR_INVALID;
  }
  for (uint32_t f = 0; f < frame_count; ++f) {
    if (!dev_frames[f]) {
      put_err(err, err_len, "frame %u is null", f);
      return FS_ERR_INVALID;
    }
    if (row_strides[f] < (size_t)width * channels) {
      put_err(err, err_len, "frame %u: row stride smaller than its row", f);
      return FS_ERR_MISMATCH;
    }
  }
  StaticLayout lay;
  plan_layout(width, height, frame_count, &lay);
  if (lay.bytes > kStaticScratchBytes) {
    put_err(err, err_len,
            "%u frames of %ux%u need %zu bytes of planes; the static scratch holds %zu (40 MiB, e.g. 8 frames of "
            "512x512)",
            frame_count, width, height, lay.bytes, kStaticScratchBytes);
    return FS_ERR_UNSUPPORTED;
  }
  unsigned char* base = nullptr;
  int rc = scratch_on_current_device(&base, err, err_len);
  if (rc != FS_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  auto fail = [&](cudaError_t e, const char* what) {
    put_err(err, err_len, "%s: %s", what, cudaGetErrorString(e));
    return FS_ERR_CUDA;
  };
  const uint32_t L = lay.L, K = frame_count;
  float* norm = (float*)(base + lay.norm);
  uint8_t* sm[32];
  float* acc[32];
  for (uint32_t l = 0; l < L; ++l) {
    sm[l] = base + lay.sm[l];
    acc[l] = (float*)(base + lay.acc[l]);
  }
  FramePlanes planes[kMaxBatch];
  const size_t n0 = (size_t)lay.pitch[0] * lay.lh[0];
  for (uint32_t k = 0; k < K; ++k) {
    planes[k].rgba = (uint32_t*)(base + lay.planes[k]);
    planes[k].w = (float*)(base + lay.planes[k] + n0 * 4);
  }
  // pass 1: weights of every frame, their sum and the support union
  RemapWeightArgs ra;
  memset(&ra, 0, sizeof(ra));
  ra.W = (int32_t)width;
  ra.H = (int32_t)height;
  ra.window_ok = (width >= contrast_window && height >= contrast_window) ? 1 : 0;
  ra.K = (int32_t)K;
  ra.accumulate = 1;
  ra.first = 1;
  ra.norm = norm;
  ra.uni = sm[0];
  ra.pitch = lay.pitch[0];
  for (uint32_t k = 0; k < K; ++k) {
    FrameIn& fi = ra.f[k];
    fi.src.px = (const uint8_t*)dev_frames[k];
    fi.src.pitch = (int64_t)row_strides[k];
    fi.src.w = (int32_t)width;
    fi.src.h = (int32_t)height;
    fi.src.ch = (int32_t)channels;
    fi.warp.kind = WARP_ALIGNED;
    ra.out[k] = planes[k];
  }
  cudaError_t e = launch_remap_weights(ra, (int)(contrast_window / 2), st);
  if (e != cudaSuccess) return fail(e, "weights launch");
  for (uint32_t l = 0; l + 1 < L; ++l) {
    MaskSupportArgs m = {sm[l],     (int32_t)lay.lw[l],     (int32_t)lay.lh[l],     lay.pitch[l],
                         sm[l + 1], (int32_t)lay.lw[l + 1], (int32_t)lay.lh[l + 1], lay.pitch[l + 1]};
    if ((e = launch_mask_support(m, st)) != cudaSuccess) return fail(e, "mask support launch");
  }
  for (uint32_t l = 0; l < L; ++l) {
    if ((e = cudaMemsetAsync(acc[l], 0, (size_t)lay.pitch[l] * lay.lh[l] * 12, st)) != cudaSuccess)
      return fail(e, "accumulator clear");
  }
  // pass 2 (one batch): level 0 from the pass-1 planes, then every level
  LevelArgs a;
  memset(&a, 0, sizeof(a));
  a.levels = (int32_t)L;
  a.K = (int32_t)K;
  a.inv_count = 1.0f / (float)K;
  a.norm = norm;
  for (uint32_t k = 0; k < K; ++k) a.in0[k] = planes[k];
  for (uint32_t l = 0; l + 1 < L || (L == 1 && l == 0); ++l) {
    a.level = (int32_t)l;
    a.wl = (int32_t)lay.lw[l];
    a.hl = (int32_t)lay.lh[l];
    a.pitch_l = lay.pitch[l];
    a.exact_expand = std::max(lay.lw[l], lay.lh[l]) <= kExactExpandMaxDim ? 1 : 0;
    a.sm_l = sm[l];
    a.acc_l = acc[l];
    a.acc_plane_l = lay.pitch[l] * lay.lh[l];
    if (l + 1 < L) {
      a.wn = (int32_t)lay.lw[l + 1];
      a.hn = (int32_t)lay.lh[l + 1];
      a.pitch_n = lay.pitch[l + 1];
      a.acc_n = acc[l + 1];
      a.acc_plane_n = lay.pitch[l + 1] * lay.lh[l + 1];
    } else {
      a.wn = a.hn = 1;
      a.pitch_n = 32;
    }
    for (uint32_t k = 0; k < K; ++k) {
      const auto slot = [&](uint32_t lv) {
        const size_t plane = (size_t)lay.pitch[lv] * lay.lh[lv];
        unsigned char* p = base + lay.slot[k][lv];
        return LevelPlanes{p, p + plane * 12, p + plane * 16, (int64_t)plane};
      };
      a.in[k] = l >= 1 ? slot(l) : LevelPlanes{};
      a.out[k] = l + 1 < L - 1 ? slot(l + 1) : LevelPlanes{};
    }
    e = l == 0 ? launch_level0(a, FS_STORAGE_F32, st) : launch_level(a, FS_STORAGE_F32, st);
    if (e != cudaSuccess) return fail(e, "level launch");
    if (L == 1) break;
  }
  // collapse straight into the caller's output
  if (L == 1) {
    e = launch_quantize(acc[0], lay.pitch[0] * lay.lh[0], lay.pitch[0], (int)width, (int)height, (uint8_t*)dev_out,
                        (int64_t)out_stride, nullptr, 0, 0, st);
    if (e != cudaSuccess) return fail(e, "quantise launch");
  }
  for (uint32_t l = L - 1; l >= 1 && L > 1; --l) {
    CollapseArgs c;
    memset(&c, 0, sizeof(c));
    c.wp = (int32_t)lay.lw[l - 1];
    c.hp = (int32_t)lay.lh[l - 1];
    c.wc = (int32_t)lay.lw[l];
    c.hc = (int32_t)lay.lh[l];
    c.pitch_p = lay.pitch[l - 1];
    c.pitch_c = lay.pitch[l];
    c.exact_expand = std::max(lay.lw[l - 1], lay.lh[l - 1]) <= kExactExpandMaxDim ? 1 : 0;
    c.acc_p = acc[l - 1];
    c.plane_p = lay.pitch[l - 1] * lay.lh[l - 1];
    c.acc_c = acc[l];
    c.plane_c = lay.pitch[l] * lay.lh[l];
    c.out = l == 1 ? (uint8_t*)dev_out : nullptr;
    c.out_pitch = (int64_t)out_stride;
    if ((e = launch_collapse(c, st)) != cudaSuccess) return fail(e, "collapse launch");
  }
  return FS_OK;
}
