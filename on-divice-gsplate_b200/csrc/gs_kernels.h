// Host-side launchers of the training-step kernels (internal to libgs_cuda).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gs_common.cuh"
#include "motion.cuh"

namespace gsk {

// ---- model layout in HBM ----
// Parameters: 4 float4 planes of `cap` slots (P[plane * cap + slot]): position + opacity
// logit, log scale + alive flag, quaternion (w, x, y, z), SH DC + 0 — the reference's
// 4 x vec4 per slot (train_common.glsl:3-8) split into planes so every access is a
// coalesced 16-byte load. SH beyond DC: `sh_stride` float planes (SH[f * cap + slot],
// f = coeff * 3 + channel). Adam moments mirror both layouts.
struct Model {
  uint32_t cap = 0, slots = 0, sh_stride = 0;
  float4* P = nullptr;
  float4* M = nullptr;
  float4* V = nullptr;
  float* SH = nullptr;
  float* MSH = nullptr;
  float* VSH = nullptr;
  float4* stats = nullptr;  // grad norm sum, visible count, max radius, abs grad sum
};

// Per (view, slot) buffers: index g = view * cap + slot.
struct ViewBuffers {
  float4* splat = nullptr;   // 3 per g: (mean xy, depth, opacity), (conic abc, radius), (rgb, clamp bits)
  float4* foot = nullptr;    // 1 per g: dilated 2D covariance abc, footprint threshold
  uint4* spans = nullptr;    // 1 per g: the footprint's tile-row spans, packed (footprint_count_spans)
  uint32_t* tiles = nullptr; // tiles touched
  uint32_t* offsets = nullptr;  // first pair, pre-sort order
  float4* grad2d = nullptr;  // 3 per g: summed pair gradients (train_pair_sum layout)
  // Atomic training steps: the projection leaves each drawn (view, slot)'s view word
  // (pack_view_word: radius and clamped-colour bits) in grad2d's unused 12th float, and the
  // optimizer reads it there instead of from the splat records.
  bool view_word = false;
  float4* dir_grad = nullptr; // 1 per slot: position gradient through the SH view direction, summed over views
};

struct StepPointers {
  const gs_frame_data* frames = nullptr;  // device: the step table's FrameData, n_views entries
  const ViewTable* vt = nullptr;          // device: the step table's view layout
  uint32_t n_views = 0;                   // fixed for a captured step
  uint32_t tile_cap = 0;                  // grids of per-tile kernels (>= any step's tiles)
  uint32_t* queue = nullptr;              // device work-queue counters, zeroed each step
  int sm_count = 148;
};

// ---- project.cu ----
// motion: non-null when some view of the step has GS_FLAG_MOTION.
void launch_project(const StepPointers& sp, const Model& m, uint32_t degree, const ViewBuffers& vb,
                    uint32_t* depth_keys, uint32_t* depth_vals, bool zero_grad2d, const Motion* motion,
                    cudaStream_t st);

// ---- sort.cu ----
struct SortScratch {
  uint32_t* hist = nullptr;           // passes x 256 (up to 8 passes: 32-bit keys at 4-bit digits)
  uint32_t* tile_counts = nullptr;    // 256 x tiles: per-tile digit counts, then the tiles' starts
  uint32_t count_tiles = 0;
  unsigned long long* scan_lookback = nullptr;
  uint32_t scan_tiles = 0;
};
constexpr uint32_t kSortTile = 256 * 15;
constexpr uint32_t kScanTile = 256 * 8;
// Sorts (keys, vals) of min(*d_count, n_max) items by key bits [0, bits), stable, in
// passes of `digit_bits` (4..8) bits. Returns true when the result ended in the alternate
// buffers.
bool radix_sort_pairs(const SortScratch& s, uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt,
                      const uint32_t* d_count, uint32_t n_max, int bits, cudaStream_t st, int* launches,
                      int digit_bits = 8);
// Exclusive scan of in[gather ? gather[k] : k] for k < n; *d_total (if non-null) = the sum.
// out must not alias in or gather (it first holds the gathered values).
void exclusive_scan(const SortScratch& s, const uint32_t* in, const uint32_t* gather, uint32_t* out, uint32_t n,
                    uint32_t* d_total, cudaStream_t st, int* launches);

// ---- pairs.cu ----
// total: the scan's total (the end of the last item's pairs).
// values: each pair's pre-sort index, or (payload_gaussian) its gaussian g, which the sort
// then carries to the raster passes directly (atomic training steps, which never need the
// pre-sort index).
void launch_emit(const StepPointers& sp, const ViewBuffers& vb, uint32_t cap, uint32_t n_items,
                 const uint32_t* sorted_vals, const uint32_t* sorted_offsets, const uint32_t* total,
                 uint32_t pair_capacity, uint32_t* keys, uint32_t* values, uint32_t* pair_gaussian, float4* pair_grads,
                 uint32_t* mismatch, bool payload_gaussian, cudaStream_t st);
// Tile ranges of the sorted pairs, and each view's span [view_span[v], view_span[kMaxViews + v])
// of them (zeroed by the caller; views without pairs keep 0, 0). With `gather` non-null,
// also sorted_g[s] = pair_gaussian[sorted_values[s]]: each sorted pair's gaussian, laid out
// in render order for the raster passes' coalesced staging.
struct PairGather {
  const uint32_t* sorted_values = nullptr;
  const uint32_t* pair_gaussian = nullptr;
  uint32_t* sorted_g = nullptr;
};
void launch_ranges(const uint32_t* sorted_keys, const uint32_t* d_count, uint32_t pair_capacity, uint2* ranges,
                   const ViewTable* vt, uint32_t* view_span, const PairGather* gather, cudaStream_t st);

// ---- raster.cu ----
struct RasterBuffers {
  const uint2* ranges = nullptr;
  const uint32_t* values = nullptr;         // per sorted pair: its pre-sort index (or g, see launch_emit)
  const uint32_t* gauss = nullptr;          // per sorted pair: its gaussian g (render order)
  float4* pixel_grad = nullptr;             // dL/dC rgb, final T
  float4* pixel_out = nullptr;              // rendered colour rgb (over the background), loss weight
  uint32_t* pixel_count = nullptr;
  uint32_t* image = nullptr;
  float* pixel_dot = nullptr;
  float* tile_loss = nullptr;               // 16 per global tile
  uint32_t* tile_count = nullptr;
  // The forward's per-warp tile sums (kTileWarpSlots warps x 16 floats per tile; slot 14
  // holds the warp's furthest last contributor as bits) and, per tile, how many of its
  // warps have written theirs (the last one adds them up and resets it to 0).
  float* tile_part = nullptr;
  uint32_t* tile_done = nullptr;
  // The SSIM gradient maps w A, w B, w C (rgb each) of every pixel, 36 bytes:
  // ssim_maps[2 p] = (A rgb, B r), ssim_maps[2 p + 1] = (B g, B b, C r, C g), ssim_last[p] = C b.
  float4* ssim_maps = nullptr;
  float* ssim_last = nullptr;
};
constexpr uint32_t kTileWarpSlots = 8;  // the most warps a tile has (one pixel per thread)
// px: pixels per thread (1, 2 or 4); batch: splats staged per round (64, 128, 256);
// async: stage the next round with cp.async while the current one blends. contributions
// (non-null): a counting launch that also adds the evaluations that blend into it.
void launch_raster_forward(const StepPointers& sp, const ViewBuffers& vb, const RasterBuffers& rb, int px, int batch,
                           bool async, unsigned long long* contributions, cudaStream_t st);
// Per-pair gradients (deterministic: pair_grads at the pre-sort index) or atomics into
// vb.grad2d (fast), staging `batch` (32 or 64) splats per round. Skipped on device when
// *d_pairs > accept.
void launch_raster_backward(const StepPointers& sp, const ViewBuffers& vb, const RasterBuffers& rb,
                            float4* pair_grads, bool deterministic, int px, int batch, bool async,
                            const uint32_t* d_pairs, uint32_t accept, cudaStream_t st);

// ---- loss.cu ----
void launch_ssim(const StepPointers& sp, const RasterBuffers& rb, cudaStream_t st);
void launch_ssim_grad(const StepPointers& sp, const RasterBuffers& rb, cudaStream_t st);
// view_sums[v * stride + 0..15]: the view's 16 tile sums; parts: scratch of
// n_views * kLossParts * 16 doubles.
constexpr uint32_t kLossParts = 16;
void launch_loss_reduce(const StepPointers& sp, const float* tile_loss, double* view_sums, uint32_t stride,
                        double* parts, cudaStream_t st);

// ---- step.cu ----
void launch_pair_sum(const ViewBuffers& vb, uint32_t n_items, const uint32_t* depth_order, const uint32_t* first,
                     const float4* pair_grads, const uint32_t* d_pairs, uint32_t accept, cudaStream_t st);
// motion: non-null when some view of the step has GS_FLAG_MOTION.
void launch_step(const StepPointers& sp, const Model& m, uint32_t degree, const ViewBuffers& vb,
                 const uint32_t* d_pairs, uint32_t accept, const Motion* motion, cudaStream_t st);
// Camera pose gradients of the views with GS_FLAG_POSE_GRAD (before launch_step, which
// updates the parameters): out[v * stride + 0..5]. partial: n_views * pose_blocks(slots) * 8.
uint32_t pose_blocks(uint32_t slots);
void launch_pose_grad(const StepPointers& sp, const Model& m, uint32_t degree, const ViewBuffers& vb,
                      const uint32_t* d_pairs, uint32_t accept, const Motion* motion, float* partial, double* out,
                      uint32_t stride, cudaStream_t st);
// Subject motion: the per-node gradient of the views with GS_FLAG_MOTION_GRAD (before
// launch_step), out[(v * kMaxMotionNodes + node) * 8 + 0..5]; partial holds
// n_views * motion_blocks(slots, sm_count) * kMaxMotionNodes * 8 floats.
uint32_t motion_blocks(uint32_t slots, int sm_count);
void launch_motion_grad(const StepPointers& sp, const Model& m, uint32_t degree, const ViewBuffers& vb,
                        const uint32_t* d_pairs, uint32_t accept, const Motion& motion, float* partial, double* out,
                        cudaStream_t st);
// Binds the slots in use to their 4 nearest nodes (train_motion_bind.comp).
void launch_motion_bind(const Model& m, const Motion& motion, cudaStream_t st);
struct DensifyScratch {
  uint32_t* spawn = nullptr;     // action per slot
  uint32_t* release = nullptr;   // 1 per freed slot
  uint32_t* wants = nullptr;     // 1 per spawning slot
  uint32_t* free_pos = nullptr;  // exclusive scans
  uint32_t* spawn_pos = nullptr;
  uint32_t* free_list = nullptr;
  uint32_t* counters = nullptr;  // [0] free, [1] spawned, [2] pruned
};
void launch_densify(const gs_frame_data* d_frame, const Model& m, const DensifyScratch& ds, const SortScratch& ss,
                    cudaStream_t st, int* launches);
void launch_reset_opacity(const Model& m, float max_logit, cudaStream_t st);

// Work-queue counters (StepPointers::queue).
constexpr int kQueueForward = 0, kQueueBackward = 1, kQueueCount = 4;

// ---- layout conversions (api.cu) ----
void launch_params_to_planes(const float* params16, const float* sh, uint32_t count, const Model& m, cudaStream_t st);
void launch_planes_to_params(const Model& m, const float4* P, const float* SH, float* params16, float* sh,
                             uint32_t count, cudaStream_t st);
void launch_projected_record(const ViewBuffers& vb, uint32_t view, uint32_t cap, uint32_t slots, float* out16,
                             cudaStream_t st);

}  // namespace gsk
