/*
 * libgs_cuda — the C ABI of the B200 (sm_100a) 3D Gaussian Splatting training step.
 *
 * It replaces the reference engine's private pass recorders and their Vulkan dispatch:
 * gs::Trainer::record_project / record_sort / record_rasterize / record_loss /
 * record_backward / record_optimize / record_scan, densify and reset_opacity
 * (engine/include/gs/trainer.h:429-443, engine/src/trainer.cpp:576-586, 665-776,
 * 1083-1128), which bind std430 buffers and call VkContext::dispatch
 * (engine/include/gs/vk_context.h:172-184). The caller keeps the reference's host code
 * above this line (gs::Trainer's public API, gs_train, gs_render).
 *
 * Conventions (the reference throws std::runtime_error / VulkanError with a message,
 * engine/include/gs/vk_context.h:18-29; here every function returns a status):
 *  - 0 is success; nonzero is one of GS_ERR_*; gs_last_error() gives the message of the
 *    calling thread's latest failure.
 *  - No device pointers cross this boundary: host pointers are copied before return.
 *  - The library owns all device memory and grows its pair buffers itself, as the
 *    reference grows them on overflow (engine/src/trainer.cpp:588-624).
 *  - One context per device and caller thread; calls on a context are serialised on its
 *    own CUDA stream and are synchronous unless stated otherwise.
 *
 * Layouts crossing the boundary are the reference's: 16 floats of parameters per slot
 * (train_common.glsl:3-8: position xyz + opacity logit, log scale xyz + alive flag,
 * quaternion w x y z, SH DC rgb + unused), `sh_stride` floats of SH beyond DC per slot
 * ([coeff][rgb]), RGBA8 images, and FrameData (train_common.glsl:15-37) per view.
 */
#ifndef GS_CUDA_H
#define GS_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_OK 0
#define GS_ERR_INVALID 1   /* invalid argument */
#define GS_ERR_NO_MEMORY 2 /* device or host allocation failed */
#define GS_ERR_CAPACITY 3  /* more pairs than the largest buffer the library will allocate */
#define GS_ERR_TIMEOUT 4   /* a bounded device-side wait gave up (no kernel of the library waits on another) */
#define GS_ERR_CUDA 5      /* any other CUDA error */

#define GS_MAX_VIEWS 16

/* Flags in gs_frame_data.model[3] (train_common.glsl:50-57). */
#define GS_FLAG_MASKED_TARGET 1u /* composite the target over the background by its alpha */
#define GS_FLAG_SSIM 4u          /* measure SSIM (and its gradient when training) */
/* Sum the gradient of the loss with respect to a small change of this view's camera pose
   (gs_step_result.pose_grad; train_step.glsl:7-10, trainer.cpp:74). */
#define GS_FLAG_POSE_GRAD 8u
/* On the first view: the step computes gradients (pose_grad) but changes neither the
   model nor its densification statistics (train_step.glsl:92-100, 222). */
#define GS_FLAG_POSE_ONLY 16u
/* The gaussians follow the subject's motion in this view (the node motions set with
   gs_set_view_motion; train_motion.glsl, train_common.glsl:55). */
#define GS_FLAG_MOTION 32u
/* Sum the loss gradient with respect to each node's motion in this view
   (gs_motion_gradient; train_step.glsl:11-17, train_common.glsl:56). */
#define GS_FLAG_MOTION_GRAD 64u
/* Most subject-motion control nodes (the reference's kMaxMotionNodes). */
#define GS_MAX_MOTION_NODES 128u
#define GS_FLAG_SPARSE_ADAM 128u /* gaussians that drew nothing keep their values and moments */

/* Per-view step constants: FrameData of train_common.glsl:15-37, filled as
   Trainer::write_frame fills it (engine/src/trainer.cpp:440-547). 288 bytes. */
typedef struct gs_frame_data {
  float rot[3][4];     /* world -> camera rotation rows (OpenCV axes); [r][3] = translation */
  float cam_pos[4];    /* camera centre, world */
  float intrinsics[4]; /* fx, fy, cx, cy */
  uint32_t image[4];   /* width, height, tiles_x, tiles_y (16x16 tiles) */
  uint32_t model[4];   /* slots in use, active SH degree, sh_stride (floats), flags */
  float background[4]; /* rgb, loss scale 1 / (3 W H) */
  float lr0[4];        /* position (x camera extent, decayed), log scale, rotation, opacity */
  float lr1[4];        /* SH DC, SH rest */
  float adam[4];       /* beta1, beta2, epsilon */
  float bias[4];       /* 1 / (1 - beta1^t), 1 / (1 - beta2^t) */
  float densify0[4];   /* grad threshold, clone max scale, prune min opacity, prune max world scale */
  float densify1[4];   /* prune max screen radius, seed (uint bits), split scale divisor */
  uint32_t limits[4];  /* set by the library: pair capacity, 0, 0, most pairs the update accepts */
  float loss[4];       /* D-SSIM weight lambda, C1, C2 */
  float head[4];       /* head region centre x, y, radius (px; 0: none), loss weight */
  float exposure[4];   /* rgb: the photo's colour times this is compared (1 / gain) */
} gs_frame_data;

typedef struct gs_context gs_context;

/* Per-view outcome of a step. losses: the per-tile sums of train_forward.comp:18-23 and
   train_ssim.comp summed over the view (Trainer::read_slot, trainer.cpp:778-795):
   [0] sum |e|, [1] sum e^2, [2] SSIM sum, [3] sum w |e|, [4] sum w SSIM, [5] sum 3 w,
   [6] head sum e^2, [7] head pixels. */
typedef struct gs_step_result {
  uint32_t n_views;
  uint32_t overflow;      /* the pairs did not fit and no retry was allowed: no update */
  uint32_t retries;       /* the step ran again after growing the pair buffers */
  uint32_t tile_mismatch; /* gaussians whose emitted tiles differed from the count (whole run) */
  uint64_t pairs[GS_MAX_VIEWS];
  double losses[GS_MAX_VIEWS][8];
  float gpu_ms; /* device time of the step (CUDA events) */
  uint32_t kernels; /* kernel launches of the step */
  /* With GS_STEP_PROFILE, device milliseconds per pass (Trainer's PassTimes,
     trainer.h:173-185): [0] project, [1] sort (depth sort, scan, emit, pair sort,
     ranges), [2] rasterize, [3] loss (SSIM and its gradient), [4] backward,
     [5] optimize (pair sum + projection backward + Adam). */
  float pass_ms[6];
  /* Per view, the rest of the tile sums (train_forward.comp:142-151; Trainer::read_slot's
     fit_): [0..2] sum R^2 rgb, [3] pixels, [4..6] sum R P rgb, with R the model's colour
     and P the photo's over the pixels where both are opaque (target alpha > 0.95,
     transmittance < 0.05); [7] pixels whose target alpha is above 0. */
  double fit[GS_MAX_VIEWS][8];
  /* Per view with GS_FLAG_POSE_GRAD (else 0): dL/dd xyz then dL/dw xyz in camera axes,
     for world -> camera [W | t] becoming [(I + [w]x) W | (I + [w]x) t + d]
     (train_step.glsl:196-203; Trainer::pose_gradient, trainer.cpp:1336-1348). */
  double pose_grad[GS_MAX_VIEWS][6];
} gs_step_result;

/* Which intermediate buffer gs_snapshot copies (Trainer::DebugSnapshot, trainer.h:302-313). */
typedef enum gs_snapshot_kind {
  GS_SNAP_PIXEL_COUNT = 0,  /* uint32 per pixel: pairs up to the last contributor */
  GS_SNAP_PIXEL_GRAD = 1,   /* 4 floats per pixel: dL/dC rgb, final transmittance */
  GS_SNAP_PROJECTED = 2,    /* 16 floats per slot (train_common.glsl:9-13) */
  GS_SNAP_TILES = 3,        /* uint32 per slot: tiles touched */
  GS_SNAP_OFFSETS = 4,      /* uint32 per slot: first pair, pre-sort order (not after an atomic training step) */
  GS_SNAP_PAIR_GRADS = 5,   /* 12 floats per pair, pre-sort order (deterministic mode) */
  GS_SNAP_PAIR_TILE = 6,    /* uint32 per pair, pre-sort order: the view's tile (not after an atomic training step) */
  GS_SNAP_RENDER_ORDER = 7, /* uint32 per pair: pre-sort index in render order (not after an atomic training step) */
  GS_SNAP_DEPTH_KEY = 8,    /* uint32 per slot: 16-bit depth key */
  GS_SNAP_IMAGE = 9,        /* RGBA8 per pixel */
  GS_SNAP_RANGES = 10,      /* 2 uint32 per tile: [start, end) in render order, view-local */
  GS_SNAP_TILE_LOSS = 11,   /* 16 floats per tile */
  GS_SNAP_PIXEL_DOT = 12,   /* float per pixel: dL/dC . colour */
  GS_SNAP_STATS = 13,       /* 4 floats per slot: densification statistics */
  GS_SNAP_PAIR_GAUSSIAN = 14, /* uint32 per pair, pre-sort order: the slot (not after an atomic training step) */
  GS_SNAP_PIXEL_OUT = 15,     /* 4 floats per pixel: rendered rgb over the background, loss weight */
  GS_SNAP_SPAWN = 16,         /* uint32 per slot after gs_densify: 0 none, 1 clone, 2 split */
  GS_SNAP_MOTION_BIND = 17,   /* 8 uint32 per slot: 4 motion nodes, their 4 weights (float bits) */
  GS_SNAP_CONTRIBUTIONS = 18  /* one uint64 (view 0): the pixel-splat evaluations that blended in the
                                 latest GS_STEP_COUNT step, all its views together */
} gs_snapshot_kind;

/* Tuning knobs (Trainer options that shape buffers and kernels; trainer.h:150-165). */
typedef struct gs_tuning {
  uint32_t min_pair_capacity; /* smallest pair buffer (TrainOptions::min_pair_capacity) */
  uint64_t initial_pairs;     /* pairs to allocate before the first count (0: 4 per slot and view) */
  uint32_t deterministic;     /* 1: per-pair gradients + fixed-order sum (bit-stable); 0: atomics */
  uint32_t forward_pixels;    /* pixels per thread in the forward pass: 1, 2 or 4 (0: default) */
  uint32_t backward_pixels;   /* pixels per thread in the backward pass: 1, 2 or 4 (a warp covers an
                                 8 x 4, 8 x 8 or 8 x 16 block of a tile), or 8 (one warp per 16 x 16
                                 tile; backward_batch does not apply) (0: default) */
  uint32_t retry;             /* 1 (default): grow the pair buffers and run again on overflow */
  uint32_t graph;             /* 1: capture the step as a CUDA graph and replay it while its launch
                                 structure (views, slots, buffer sizes, SH degree, mode) holds */
  uint32_t backward_batch;    /* splats staged per round of the deterministic backward: 32 or 64
                                 (0: default); the fast backward stages 32 per warp */
  uint32_t sort_digit_bits;   /* radix digit width of the depth and pair sorts: 4..8 (0: default 8) */
  uint32_t forward_batch;     /* splats staged per round of the forward pass with stage_async: 64, 128 or
                                 256 (0: default 256); without it each warp stages 32 per round */
  uint32_t tune_reduction;    /* 1: gs_autotune may also switch `deterministic` (0: it keeps the caller's) */
  uint32_t stage_async;       /* 1: raster passes copy the next round of splats with cp.async while the
                                 current one blends (double-buffered; the forward and the
                                 deterministic backward); 0: plain loads */
} gs_tuning;

typedef struct gs_model_info {
  uint32_t capacity, slots, sh_stride;
  uint64_t pair_capacity;
  uint64_t device_bytes;
} gs_model_info;

/* Message of the calling thread's latest failure ("" if none). */
const char* gs_last_error(void);

/* Context on CUDA device `device`: the role of the VkContext& the reference's Trainer
   takes (trainer.h:253), device + stream owner. */
int gs_create(int device, gs_context** out);
int gs_destroy(gs_context* ctx);

/* Parameters and Adam state: the Trainer constructor's upload (trainer.cpp:388-417).
   capacity slots are allocated; `count` are initialised from params16 (16 floats per
   slot) and sh (sh_stride floats per slot, may be NULL when sh_stride is 0). Moments and
   statistics start at zero. */
int gs_model_init(gs_context* ctx, uint32_t capacity, uint32_t sh_stride, const float* params16, const float* sh,
                  uint32_t count);
int gs_model_info_get(gs_context* ctx, gs_model_info* out);
/* The slots in use, in the reference layout (Trainer::export_scene, trainer.cpp:1773-1800
   reads the same buffers). Either pointer may be NULL. */
int gs_model_export(gs_context* ctx, float* params16, float* sh, uint32_t max_slots, uint32_t* slots);
/* Adam moments of the slots in use (Trainer::first_step_gradients, trainer.cpp:1802-1811,
   divides m by 1 - beta1). Any pointer may be NULL. */
int gs_model_moments(gs_context* ctx, float* m16, float* v16, float* m_sh, float* v_sh);

/* The views of the next step: one FrameData each, with its own resolution, and each
   view's target image (RGBA8, width x height x 4 bytes; NULL: no loss). Replaces
   Trainer::write_frame's host-visible uploads (trainer.cpp:440-547, 1024-1031). The
   targets are copied asynchronously on a second stream of the context, overlapping the
   next step's projection and sort: their buffers must stay unchanged until the next
   gs_step returns (pinned memory is copied by DMA). */
int gs_set_views(gs_context* ctx, uint32_t n_views, const gs_frame_data* frames, const uint8_t* const* rgba_targets);

/* Target images kept in HBM across steps (the dataset's views): n_images RGBA8 images of
   widths[i] x heights[i]. Replaces the per-step target uploads of Trainer::run_batch
   (trainer.cpp:1024-1031) for callers that train on a fixed dataset. */
int gs_dataset_set(gs_context* ctx, uint32_t n_images, const uint32_t* widths, const uint32_t* heights,
                   const uint8_t* const* rgba);
/* As gs_set_views, with view v's target the dataset image images[v] (same size). */
int gs_set_views_dataset(gs_context* ctx, uint32_t n_views, const gs_frame_data* frames, const uint32_t* images);

#define GS_STEP_TRAIN 1u   /* backward pass and Adam (else: forward and loss only) */
#define GS_STEP_PROFILE 2u /* time each pass with CUDA events (pass_ms) */
#define GS_STEP_COUNT 4u   /* count the evaluations that blend (GS_SNAP_CONTRIBUTIONS); runs without
                              the step's graph, so time no step that counts */

/* One step over the views set by gs_set_views: project -> key build + sort -> tile ranges
   -> rasterise -> L1 + SSIM -> backward -> Adam (trainer.cpp:825-831). With more than one
   view, the views' gradients are summed and one Adam step is taken. Overflowing pair
   buffers are grown and the step re-run (trainer.cpp:814-836) unless tuning.retry is 0. */
int gs_step(gs_context* ctx, uint32_t flags, gs_step_result* out);

/* Forward only: `frame`'s view of the model as RGBA8 (alpha = coverage) into rgba_out
   (Trainer::render_with, trainer.cpp:1140-1153). */
int gs_render(gs_context* ctx, const gs_frame_data* frame, uint8_t* rgba_out);

/* Adaptive density control with `frame`'s thresholds (Trainer::densify,
   trainer.cpp:1083-1119; train_densify_mark.comp, train_densify_spawn.comp). Slots are
   placed deterministically (free list in slot order, spawners in slot order). counters:
   [0] free slots, [1] gaussians that asked to spawn, [2] pruned, [3] slots in use after. */
int gs_densify(gs_context* ctx, const gs_frame_data* frame, uint32_t counters_out[4]);

/* Caps every opacity logit at max_logit and clears its moments
   (Trainer::reset_opacity, trainer.cpp:1121-1128). */
int gs_reset_opacity(gs_context* ctx, float max_logit);

/* Copies an intermediate buffer of the latest step's view `view` to host (the reference's
   Trainer::debug_snapshot, trainer.cpp:1813-1852). `needed` receives the byte size;
   host may be NULL to query it. */
int gs_snapshot(gs_context* ctx, uint32_t view, gs_snapshot_kind which, void* host, size_t bytes, size_t* needed);

int gs_set_tuning(gs_context* ctx, const gs_tuning* tuning);
int gs_get_tuning(gs_context* ctx, gs_tuning* tuning);

/* Picks the tuning for the views set last (gs_set_views / gs_set_views_dataset, with
   targets), as Trainer's backward retune does (trainer.h:150-157; trainer.cpp:876-897, 983-987): it
   times training steps under candidate settings of forward_pixels, (backward_pixels,
   backward_batch) and sort_digit_bits, one knob after the other keeping the fastest (each
   candidate: one untimed step, then `steps_per_candidate` steps timed with CUDA events),
   and makes the fastest the context's tuning (written to `chosen` when not NULL). The
   candidates compute the same gradients up to summation order. The model, its moments and
   densification statistics are restored afterwards, so the call leaves training where it
   was; it needs device memory for one copy of them. */
int gs_autotune(gs_context* ctx, uint32_t steps_per_candidate, gs_tuning* chosen);

/* Subject motion (SC-GS; train_motion.glsl, train_motion_bind.comp, Trainer's motion state,
   trainer.cpp:1398-1690). The model stays the subject at rest; in a view with
   GS_FLAG_MOTION each control node k moves rigidly (x -> R_k x + b_k) and every slot
   follows its 4 nearest nodes, blended by weight.
   gs_motion_nodes: the nodes at rest, count <= GS_MAX_MOTION_NODES, 4 floats each
   (position xyz, 1 / (2 r^2) with r the node's radius); binds every slot in use to its 4
   nearest nodes with weights exp(-d^2 / (2 r^2)) normalised (the nearest alone when all
   underflow). count 0 removes them. gs_model_init removes them too; gs_densify re-binds. */
int gs_motion_nodes(gs_context* ctx, uint32_t count, const float* nodes4);
/* Binds the slots in use again (train_motion_bind.comp), for gaussians that moved. */
int gs_motion_bind(gs_context* ctx);
/* Node motions for view `view` (< GS_MAX_VIEWS) of the next steps, 20 floats per node:
   the 3 rows of [R | b] (b = c - R n), the turn vector (xyz, 0) and the moved position c
   (xyz, 0). gs_render uses view 0's. Kept until set again. */
int gs_set_view_motion(gs_context* ctx, uint32_t view, const float* nodes20);
/* After a training step whose view `view` had GS_FLAG_MOTION_GRAD: per node (count of
   them) dL/dshift xyz then dL/dturn xyz in world axes, summed over the slots
   (train_step.glsl:270-337, train_motion_sum.comp). */
int gs_motion_gradient(gs_context* ctx, uint32_t view, double* out, uint32_t count);

/* No counterpart in the reference. For callers that cannot allocate device memory —
   runtimes whose pool owns all device memory and forbids allocations outside it, plugins
   that get only the buffers such a runtime passes them, loops that cannot afford an
   allocation's device synchronisation — this sorts n (key, value) pairs already in device
   memory, in place, stably by key bits [0, key_bits), with the library's radix sort, and
   allocates nothing: its scratch is a static device array sized for
   GS_SORT_NOALLOC_MAX_ITEMS pairs (about 8.3 MB, held by every GPU that loads the library
   until exit). Larger n is rejected with GS_ERR_INVALID.
   - `stream` is a cudaStream_t (NULL: the legacy default stream) on the current device;
     the call returns after the sort has finished on it.
   - The first call on a device looks up the scratch's device address (set-up, once per
     device, with that device current); make that first call before any stream capture.
   - Every call shares the one array: calls that overlap on the GPU (other streams, other
     host threads on the same device) race and corrupt each other's results. */
#define GS_SORT_NOALLOC_MAX_ITEMS (1u << 20)
int gs_sort_pairs_noalloc(uint32_t* keys, uint32_t* values, uint32_t n, uint32_t key_bits, void* stream);

#ifdef __cplusplus
}
#endif

#endif
