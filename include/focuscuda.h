/*
 * focuscuda.h - C ABI of libfocuscuda.so, the sm_100a (B200) implementation
 * of the focus-stacker remap + pyramid-contrast fusion hot path.
 *
 * Plain C types only: pointers, sizes, PODs.  Every call returns an fs_status
 * (0 = FS_OK); fs_last_error() gives a message for the last failure on a
 * context.  Pixel buffers are interleaved, row-major, u8 or u16 samples
 * (fs_stack_desc.sample_bits), with an explicit row stride in bytes.
 *
 * Each entry point names the reference (asingleoat/focus-stacker, Zig)
 * interface it replaces; paths are relative to the reference project root.
 */
#ifndef FOCUSCUDA_H
#define FOCUSCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FS_API_VERSION 1

typedef enum fs_status {
  FS_OK = 0,
  FS_ERR_INVALID = 1,     /* bad argument (size, window, null pointer, ...)  */
  FS_ERR_OOM = 2,         /* device or pinned host allocation failed         */
  FS_ERR_BUDGET = 3,      /* request exceeds the context's HBM budget        */
  FS_ERR_CUDA = 4,        /* CUDA runtime error                              */
  FS_ERR_TIMEOUT = 5,     /* a bounded device wait gave up                   */
  FS_ERR_STATE = 6,       /* call out of order (e.g. frame after finish)     */
  FS_ERR_MISMATCH = 7,    /* frame size / format differs from the stack's    */
  FS_ERR_UNSUPPORTED = 8, /* valid but not implemented (e.g. 16-bit FP16 levels) */
  FS_ERR_NO_DEVICE = 9    /* no CUDA device / library built for another arch */
} fs_status;

/* == ImagePose (src/optimize.zig:32-48), same field order and defaults
 * (base_hfov_degrees = 50).  Angles in radians, hfov in degrees. */
typedef struct fs_pose {
  double yaw, pitch, roll, hfov_delta;
  double trans_x, trans_y, trans_z;
  double translation_plane_yaw, translation_plane_pitch;
  double radial_a, radial_b, radial_c;
  double center_shift_x, center_shift_y;
  double base_hfov_degrees;
} fs_pose;

/* == remap.Rect (src/remap.zig:573-578): [left, right) x [top, bottom). */
typedef struct fs_rect {
  int32_t left, top, right, bottom;
} fs_rect;

typedef struct fs_ctx fs_ctx;
typedef struct fs_stack fs_stack;

/* Pyramid level storage for the precision forms. */
typedef enum fs_level_storage { FS_STORAGE_F32 = 0, FS_STORAGE_F16 = 1, FS_STORAGE_BF16 = 2 } fs_level_storage;

/* ---------------------------------------------------------------- context */

/* Open a context on CUDA device `device`.  hbm_budget_bytes caps the device
 * memory the context may hold (0 = half of the device's free memory, the
 * analogue of --memory-fraction 0.5, src/memory_budget.zig:3-53). */
int fs_create(int device, uint64_t hbm_budget_bytes, fs_ctx** out);
void fs_destroy(fs_ctx* ctx);
const char* fs_last_error(const fs_ctx* ctx);
const char* fs_status_string(int status);
int fs_api_version(void);
/* Bytes of device memory in the context's live buffers (what its budget
 * counts). */
uint64_t fs_ctx_device_bytes(const fs_ctx* ctx);
/* The context's HBM budget in bytes (0 for a null context).  Not part of the
 * reference. */
uint64_t fs_ctx_budget(const fs_ctx* ctx);
/* Wait for all work queued on the context's stream. */
int fs_ctx_synchronize(fs_ctx* ctx);
/* Buffers come from a stream-ordered memory pool shared by the contexts of
 * the process on a device (allocation and release never synchronise the
 * device); memory of destroyed stacks stays cached in the pool for later
 * stacks.  fs_ctx_trim waits for the context's streams and returns the
 * cached memory to the device.  Not part of the reference. */
int fs_ctx_trim(fs_ctx* ctx);
/* Grow the shared pool's cache by `bytes` (allocate and release), so that
 * later stacks find their memory without growing the pool; for a serving
 * process that takes its HBM budget up front.  Not part of the reference. */
int fs_ctx_reserve(fs_ctx* ctx, uint64_t bytes);
/* Change the context's HBM budget (later allocations and pass-2 mode choices
 * use it; memory already held is not released).  Used by a serving loop that
 * hands each admitted stack its reservation.  Not part of the reference. */
int fs_ctx_set_budget(fs_ctx* ctx, uint64_t hbm_budget_bytes);
/* Level schedule of the split-pyramid stacks begun on the context from now
 * on (and of the stacks of batches created from it): levels l >= 1 of at
 * least fuse_min_tiles 64x32 tiles blend and REDUCE their masks in one pass
 * (0: 1184; UINT32_MAX: none), and the levels whose sides are both at most
 * tail_side (0: 64, at most 64) run as the small-level tail.  Every schedule
 * gives the same bytes; the batched form's autotuner picks among them.  Not
 * part of the reference. */
int fs_ctx_set_level_schedule(fs_ctx* ctx, uint32_t fuse_min_tiles, uint32_t tail_side);
/* out[i] = w[i] / n[i] (device arrays of `count` floats) as the level-0
 * blend of the split pyramid divides each frame's weight by the weight sum:
 * Markstein's refinement from n's correctly rounded reciprocal, which the
 * blend forms once per pixel for all frames.  For tests that compare it bit
 * for bit with the IEEE division.  No counterpart in the reference (which
 * divides, src/fuse/pyramid.zig:303-316). */
int fs_check_normalise(fs_ctx* ctx, const float* w, const float* n, float* out, size_t count);
/* The CUDA stream (cudaStream_t) all of the context's kernels run on, for
 * callers that order their own work or record events against it. */
int fs_ctx_stream(const fs_ctx* ctx, void** stream);
/* Kernel accounting: number of kernels this context launched so far, and
 * (when timing is enabled) per-kernel launch counts and device time measured
 * with CUDA events on the launching stream.  Kernel names: "pass1",
 * "remap_weights" (pass-2 re-remap), "level0", "level", "collapse",
 * "mask_support", "remap".  Enabling or
 * disabling timing clears the recorded times.  Not part of the reference. */
uint64_t fs_ctx_launch_count(const fs_ctx* ctx);
int fs_ctx_set_kernel_timing(fs_ctx* ctx, int enable);
int fs_ctx_kernel_stats(fs_ctx* ctx, const char* kernel, uint64_t* launches, double* total_ms);

/* ------------------------------------------------- host pose utilities */

/* Fill *pose with ImagePose defaults (all zero, base_hfov_degrees = 50). */
void fs_pose_default(fs_pose* pose);

/* Common-overlap ROI of the active frames (FP64, host):
 * replaces remap.computeCommonOverlapRoi, src/remap.zig:585-633.
 * *has_roi = 0 when the frames share no overlap (the reference's null). */
int fs_compute_roi(const fs_pose* poses, const uint32_t* widths, const uint32_t* heights, const uint8_t* active,
                   size_t n, fs_rect* out, int* has_roi);

/* Map n aligned-frame points (x, y pairs) to source-frame coordinates with
 * the per-frame transform this library composes on the host in FP64 (the
 * map the kernels evaluate): replaces optimize.inverseTransformPointCached,
 * src/optimize.zig:3593-3616. */
int fs_inverse_map_points(const fs_pose* pose, uint32_t width, uint32_t height, size_t n, const double* xy,
                          double* out_xy);

/* Forward map of n source-frame points to aligned-frame coordinates (FP64,
 * host): replaces optimize.transformPoint, src/optimize.zig:3506-3525
 * ((-1, -1) where the reference's chain rejects the point). */
int fs_forward_map_points(const fs_pose* pose, uint32_t width, uint32_t height, size_t n, const double* xy,
                          double* out_xy);

/* Normaliser of the no-wrap EXPAND at output (x, y) for a src_w x src_h
 * source level, as the kernels evaluate it: the position-dependent divisors
 * of expandRgbExactNoWrap, src/fuse/pyramid.zig:1167-1354 (host only). */
float fs_exact_expand_divisor(int x, int y, int src_w, int src_h);

/* ------------------------------------------------------------- remap only */

/* Remap one frame through its pose into the ROI with a support-alpha
 * channel: replaces remap.remapRigidImage, src/remap.zig:166-204 (u8).
 * src: width x height x channels (1 or 3) samples; dst: roi-sized,
 * (channels + 1) samples per pixel.  roi == NULL means the full frame.
 * Host buffers; the call copies in and out and returns when done. */
int fs_remap_frame(fs_ctx* ctx, const void* src, size_t src_stride, uint32_t width, uint32_t height,
                   uint32_t channels, const fs_pose* pose, const fs_rect* roi, void* dst, size_t dst_stride);

/* Same, with device pointers (src and dst already in device memory). */
int fs_remap_frame_device(fs_ctx* ctx, const void* src, size_t src_stride, uint32_t width, uint32_t height,
                          uint32_t channels, const fs_pose* pose, const fs_rect* roi, void* dst, size_t dst_stride);

/* The u16 twins: 16-bit samples in and out, alpha 65535 inside the frame and
 * round(support * 65535) on its edge; replaces remap.remapRigidImage on u16
 * images (remapU16, src/remap.zig:280-336, 443-541, 841-937).  Strides in
 * bytes. */
int fs_remap_frame16(fs_ctx* ctx, const void* src, size_t src_stride, uint32_t width, uint32_t height,
                     uint32_t channels, const fs_pose* pose, const fs_rect* roi, void* dst, size_t dst_stride);
int fs_remap_frame16_device(fs_ctx* ctx, const void* src, size_t src_stride, uint32_t width, uint32_t height,
                            uint32_t channels, const fs_pose* pose, const fs_rect* roi, void* dst,
                            size_t dst_stride);

/* ---------------------------------------------------------------- JPEG */

/* Size of a JPEG file the decoder takes (FS_ERR_UNSUPPORTED otherwise: a
 * progressive, arithmetic-coded, 12-bit, grayscale or otherwise subsampled
 * file).  Host only. */
int fs_jpeg_info(const void* data, size_t len, uint32_t* width, uint32_t* height);

/* Decode a JPEG file to interleaved RGB u8 (device_dst != 0: dst is device
 * memory), the image libjpeg's default decompression gives (image_io.loadImage,
 * src/image_io.zig:160-173).  Returns when the image is in dst. */
int fs_decode_jpeg(fs_ctx* ctx, const void* data, size_t len, void* dst, size_t dst_stride, int device_dst);

/* ------------------------------------------------------- fusion (stacks) */

typedef struct fs_stack_desc {
  uint32_t src_width, src_height; /* input frame size                                 */
  int32_t has_roi;                /* 0: output = full frame; 1: output = roi          */
  fs_rect roi;                    /* output region in aligned-frame coordinates       */
  uint32_t channels;              /* 3 = RGB source frames; aligned input: 3 or 4     */
  uint32_t sample_bits;           /* 8 (u8) or 16 (u16; FP32 levels, output u16)     */
  uint32_t frame_count;           /* active frames that will be added (N)             */
  uint32_t contrast_window;       /* odd >= 3, default 5 (--contrast-window-size)     */
  int32_t input_is_aligned;       /* 1: frames are pre-aligned (focus_fuse_zig path)  */
  int32_t level_storage;          /* fs_level_storage                                 */
  uint32_t frames_per_batch;      /* K frames per pass over per-pixel state; 0 = auto */
} fs_stack_desc;

/* Start a pyramid-contrast fusion of frame_count frames (device state:
 * weight sums, union support, FP32 accumulator pyramid).  Replaces the
 * pass-1 set-up of stack/pipeline.zig:412-459 / fuse/pipeline.zig:292-321. */
int fs_stack_begin(fs_ctx* ctx, const fs_stack_desc* desc, fs_stack** out);

/* Pass 1 for the next active frame, in the reference's frame order: remap
 * (unless aligned) -> local-contrast weight -> alpha -> weight sum and
 * union support.  Replaces the body of src/stack/pipeline.zig:412-477
 * (src/fuse/pipeline.zig:292-334 for aligned input).  `pixels` is a host
 * buffer copied before the call returns; `pose` is ignored for aligned input. */
int fs_stack_add_frame(fs_stack* stack, const void* pixels, size_t row_stride, const fs_pose* pose);

/* fs_stack_add_frame without waiting for the upload: the copy is queued and
 * the call returns, so that a stack's uploads run back to back.  The host
 * buffer (best pinned) must stay valid and unchanged until fs_stack_finish
 * or fs_stack_wait has returned. */
int fs_stack_add_frame_async(fs_stack* stack, const void* pixels, size_t row_stride, const fs_pose* pose);

/* A frame given as a JPEG file (baseline sequential Huffman, 8-bit YCbCr at
 * 4:4:4, 4:2:2 or 4:2:0): decoded on the device into the stack's frame buffer
 * and run through pass 1.  Replaces image_io.loadImage of a JPEG frame
 * (src/image_io.zig:160-173) before remapRigidImage: the pixels are those
 * libjpeg gives with its default settings (islow IDCT, fancy upsampling).
 * Files with restart markers are entropy-decoded on the GPU (one thread per
 * restart interval), others on the host.  The file buffer may be reused when
 * the call returns.  A corrupt stream is reported by fs_stack_finish. */
int fs_stack_add_frame_jpeg(fs_stack* stack, const void* data, size_t len, const fs_pose* pose);

/* Same with a device pointer; the buffer must stay valid and unchanged until
 * fs_stack_finish returns (pass 2 reads it again). */
int fs_stack_add_frame_device(fs_stack* stack, const void* dev_pixels, size_t row_stride, const fs_pose* pose);

/* Pass-2 source for frames the stack could not keep in device memory: set
 * *pixels / *row_stride to host memory holding frame `frame_index` again
 * (the reference re-decodes, src/stack/pipeline.zig:561-597).  Return 0 on
 * success. */
typedef int (*fs_frame_fetch_cb)(void* user, uint32_t frame_index, const void** pixels, size_t* row_stride);

/* Pass 2 (normalise, mask + Laplacian pyramids, weighted blend) and the
 * collapse + quantise, writing interleaved RGB u8 to host memory.  Replaces
 * runPyramidStackFusion's pass 2 plus pyramid.collapseToImageWithJobsAndDebug
 * (src/stack/pipeline.zig:515-597, src/fuse/pyramid.zig:223-269). */
int fs_stack_finish(fs_stack* stack, fs_frame_fetch_cb refetch, void* user, void* out_pixels, size_t out_stride);

/* Same with a device output buffer. */
int fs_stack_finish_device(fs_stack* stack, fs_frame_fetch_cb refetch, void* user, void* dev_out, size_t out_stride);

/* fs_stack_finish without the wait: pass 2, the collapse and the copy of the
 * fused image into `out_pixels` (pinned host memory, or any host memory the
 * caller keeps alive) are queued on the context's stream and the call
 * returns; fs_stack_wait blocks until the image is in `out_pixels`.  The next
 * stack of the same context can be begun and fed meanwhile, so that its
 * frame uploads overlap this stack's pass 2 (the reference fuses stacks one
 * after another; this is the pipelined form of fs_stack_finish).
 * fs_stack_destroy waits for this stack's work only. */
int fs_stack_finish_async(fs_stack* stack, fs_frame_fetch_cb refetch, void* user, void* out_pixels,
                          size_t out_stride);
int fs_stack_wait(fs_stack* stack);

/* Optional: also write the collapsed level-0 base before quantisation
 * (interleaved RGB FP32, device memory, row stride in elements) during
 * finish.  Used to measure error against FP64 evaluations on the 16-bit
 * grid.  Not part of the reference. */
int fs_stack_set_base_output(fs_stack* stack, float* dev_base, size_t row_stride_elems);

/* Where pass 2 of the stack takes its frames from, chosen by fs_stack_begin
 * from the HBM budget: 0 = pass-1 planes kept on the device (remapped RGBA +
 * weight per frame, the reference's cached path), 1 = frames kept on the
 * device and remapped again, 2 = frames fetched again through the finish
 * callback and remapped again. */
int fs_stack_pass2_mode(const fs_stack* stack);

/* Device bytes a stack of `desc` holds over its life when `available_bytes`
 * of budget are free, and the pass-2 mode it would pick there (0 cache, 1
 * resident, 2 refetch, 3 laps, 4 fused); host_frames != 0 counts the upload staging ring.
 * FS_ERR_BUDGET when not even the refetch mode fits.  Allocates nothing; the
 * admission test of a serving loop (the analogue of --memory-fraction,
 * src/memory_budget.zig:3-53, applied per request).  Not part of the
 * reference. */
int fs_stack_footprint(const fs_stack_desc* desc, uint64_t available_bytes, int host_frames, uint64_t* bytes,
                       int* mode);
/* Device bytes of a stack of `desc` in pass-2 mode pass2_mode (0 cache, 1
 * resident, 2 refetch, 3 laps: the split pyramid built in pass 1, 4 fused:
 * the split pyramid with level 0 blended by the remap kernel itself, about
 * half the bytes per frame-pixel of laps), and fs_stack_begin with that mode imposed
 * (-1: chosen from the budget as fs_stack_begin does); for a caller that
 * trades memory for speed itself (a serving loop keeps more stacks in flight
 * with the cache mode than with laps).  Not part of the reference. */
int fs_stack_mode_bytes(const fs_stack_desc* desc, int pass2_mode, int host_frames, uint64_t* bytes);
int fs_stack_begin_mode(fs_ctx* ctx, const fs_stack_desc* desc, int pass2_mode, fs_stack** out);

/* Fusion method of the stack (Method, src/fuse/config.zig:10-24):
 * FS_METHOD_PYRAMID_CONTRAST (the default) or
 * FS_METHOD_HYBRID_PYRAMID_CONTRAST, the pyramid-contrast image merged with
 * the hardmask-contrast image at pyramid levels 2..5 with weight
 * hybrid_sharpness in [0, 1] (--hybrid-sharpness, default 0.35): replaces the
 * hybrid branch of src/stack/pipeline.zig:177-236 (runRemappedSinglePass +
 * mergeHybridImages, src/fuse/pyramid.zig:271-301).  Call before the first
 * frame; the hybrid method takes 8-bit samples and no frame shards. */
enum { FS_METHOD_PYRAMID_CONTRAST = 0, FS_METHOD_HYBRID_PYRAMID_CONTRAST = 1 };
int fs_stack_set_method(fs_stack* stack, int method, float hybrid_sharpness);

/* Output size of the stack (the ROI). */
int fs_stack_output_size(const fs_stack* stack, uint32_t* width, uint32_t* height);

int fs_stack_destroy(fs_stack* stack);

/* Frame-sharded stacks (not part of the reference).  A stack split over
 * several GPUs holds a contiguous shard of the frames on each; finish then
 * runs in phases with two exchanges between them:
 *   fs_stack_set_frame_total(s, N)   N = frames of the whole stack (the mask
 *                                    fallback 1/N of src/fuse/pyramid.zig:303-316)
 *   fs_stack_end_pass1(s)            pass 1 of the shard's frames done;
 *     -> sum the FS_BUFFER_WEIGHT_SUM buffers and take the maximum of the
 *        FS_BUFFER_UNION buffers over all shards, in place (e.g. NCCL);
 *   fs_stack_blend(s, refetch, user) pass 2 of the shard's frames into the
 *                                    accumulators (FS_BUFFER_ACCUMULATOR, one
 *                                    per level, 3 planes of pitch x height f32);
 *     -> sum the accumulators of all shards into one stack's;
 *   fs_stack_collapse(s, out, stride, device_out)  on that stack.
 * fs_stack_finish is the three phases with no exchange.  The sums over
 * shards change the order of the FP32 additions, so results match a single
 * stack to rounding, not bit for bit (the remap and the alpha do not
 * change). */
enum { FS_BUFFER_WEIGHT_SUM = 0, FS_BUFFER_UNION = 1, FS_BUFFER_ACCUMULATOR = 2, FS_BUFFER_HARD = 3 };
int fs_stack_set_frame_total(fs_stack* stack, uint32_t frame_total);
int fs_stack_end_pass1(fs_stack* stack);
int fs_stack_blend(fs_stack* stack, fs_frame_fetch_cb refetch, void* user);
int fs_stack_collapse(fs_stack* stack, void* out_pixels, size_t out_stride, int device_out);
/* Device buffer `which` (level: accumulators only; 0 otherwise), its bytes,
 * row pitch in elements and size.  FS_BUFFER_HARD (hybrid method): per pixel
 * the RGBA word (R | G << 8 | B << 16 | A << 24) of the hardmask winner. */
int fs_stack_buffer(fs_stack* stack, int which, uint32_t level, void** ptr, uint64_t* bytes, int64_t* pitch,
                    uint32_t* width, uint32_t* height);

/* One-shot form over host frames already in memory: begin, add every frame
 * in order, finish.  Replaces runCollapsedPyramidStackPass
 * (src/stack/pipeline.zig:314-359) / runCollapsedPyramidPass
 * (src/fuse/pipeline.zig:148-180). */
int fs_fuse_stack(fs_ctx* ctx, const fs_stack_desc* desc, const void* const* frames, const size_t* row_strides,
                  const fs_pose* poses, void* out_pixels, size_t out_stride);

/* No counterpart in the reference.  Fuse-only fusion (the result of
 * fs_fuse_stack with input_is_aligned = 1) of 1..8 pre-aligned RGB / RGBA u8
 * frames already on the current device, written as RGB u8 into dev_out, with
 * every intermediate plane in a file-scope device array of 40 MiB (8 frames
 * of 512 x 512 fit; larger stacks are rejected with FS_ERR_UNSUPPORTED).
 * Needs no context and allocates no device memory, for callers that must not
 * allocate while they run.  The work is queued on `stream` (cudaStream_t of
 * the current device, NULL = default stream) and the call returns without
 * waiting for it.  The first call on a device loads the module there (the
 * set-up; make it before any stream capture); every call looks the array's
 * address up again in the current context, so a reset device or another
 * context never gets a stale address.  The 40 MiB are reserved on a device
 * when the module loads there (at the first static call with lazy module
 * loading, at context creation with CUDA_MODULE_LOADING=EAGER) and lie outside
 * every fs_ctx budget.  Every
 * call in the process shares the array: calls must not overlap in time on the
 * device (order them on one stream or with events), or they corrupt each
 * other's planes.  A message for a failure goes to err (err_len bytes, may be
 * NULL). */
int fs_fuse_aligned_device_static(const void* const* dev_frames, const size_t* row_strides, uint32_t frame_count,
                                  uint32_t width, uint32_t height, uint32_t channels, uint32_t contrast_window,
                                  void* dev_out, size_t out_stride, void* stream, char* err, size_t err_len);

/* ---------------------------------------------------------------- batches */

/* Batched form (not part of the reference): n independent stacks over
 * frames already in device memory, fused together.  Stack i has desc[i],
 * frames[i][0 .. frame_count-1] (device pointers, row stride row_strides[i]),
 * poses[i] (NULL list for aligned input) and a device RGB u8 output
 * dev_out[i] (row stride out_strides[i]).  The stacks are spread over `lanes`
 * streams, largest first to the least-loaded lane; the stacks of a lane run
 * one after another and share one device arena the size of the lane's
 * largest stack, held for the life of the batch and counted against ctx's
 * budget.  pass2_mode: 3 split pyramid (LAPS), 4 split pyramid with level 0
 * fused into pass 1, 0 cached pass-1 planes, 1 frames kept and remapped
 * again (stacks of fewer than three levels take 0 in modes 3 and 4); -1
 * takes the first of 3, 4, 0, 1 whose arenas fit the budget.  The first
 * fs_batch_run
 * executes the work directly; the second captures the same launches into a
 * CUDA graph, which every later run replays with one graph launch, reading
 * the frames at the same addresses (refill them in place between runs).
 * Each run returns when every output is written. */
typedef struct fs_batch fs_batch;
int fs_batch_create(fs_ctx* ctx, uint32_t n, const fs_stack_desc* descs, const void* const* const* frames,
                    const size_t* row_strides, const fs_pose* const* poses, void* const* dev_out,
                    const size_t* out_strides, uint32_t lanes, int pass2_mode, fs_batch** out);
int fs_batch_run(fs_batch* batch);
int fs_batch_stack_count(const fs_batch* batch);
/* Pass-2 mode of stack i (0 cache, 1 resident, 3 laps, 4 fused). */
int fs_batch_pass2_mode(const fs_batch* batch, uint32_t i);
/* 1 once runs replay a captured graph. */
int fs_batch_uses_graph(const fs_batch* batch);
int fs_batch_destroy(fs_batch* batch);

/* ------------------------------------------------------ synthetic input */

/* Render frame k of a synthetic focus stack (seeded; see the generator in
 * the library source) directly into device memory as interleaved RGB u8,
 * and return the pose that realigns it.  scene: 0 = small (blur <= 3 px,
 * shifts +-20 px, roll +-0.2 deg), 1 = production (blur <= 8 px, shifts +-60
 * px, roll +-0.3 deg).  Not part of the reference; used by tests and the
 * benchmark. */
int fs_synth_frame_device(fs_ctx* ctx, uint64_t seed, int scene, uint32_t width, uint32_t height, uint32_t frame,
                          uint32_t frame_count, void* dev_out, size_t out_stride, fs_pose* pose_out);

/* Pose of synthetic frame k (host only). */
int fs_synth_pose(uint64_t seed, int scene, uint32_t width, uint32_t height, uint32_t frame, uint32_t frame_count,
                  fs_pose* pose_out);

#ifdef __cplusplus
}
#endif

#endif /* FOCUSCUDA_H */
