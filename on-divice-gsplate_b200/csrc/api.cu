// The C ABI of libgs_cuda (include/gs_cuda.h): device memory, the step's launch sequence
// and the overflow protocol. Replaces Trainer::record_* and VkContext::run
// (engine/src/trainer.cpp:576-776, engine/src/vk_context.cpp:583-632).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gs_kernels.h"

namespace {

thread_local std::string g_last_error;

struct Failure {
  int code;
  std::string message;
};

#define GS_CUDA_TRY(expr)                                                                                  \
  do {                                                                                                     \
    const cudaError_t e_ = (expr);                                                                         \
    if (e_ != cudaSuccess)                                                                                 \
      throw Failure{e_ == cudaErrorMemoryAllocation ? GS_ERR_NO_MEMORY : GS_ERR_CUDA,                     \
                    std::string(#expr) + ": " + cudaGetErrorString(e_)};                                   \
  } while (0)

template <typename F>
int guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return GS_OK;
  } catch (const Failure& e) {
    g_last_error = e.message;
    return e.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return GS_ERR_INVALID;
  }
}

[[noreturn]] void fail(int code, const std::string& msg) { throw Failure{code, msg}; }

template <typename T>
void dev_alloc(T*& p, size_t count) {
  if (p) cudaFree(p);
  p = nullptr;
  if (count == 0) count = 1;
  GS_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T)));
}
template <typename T>
void dev_free(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

uint32_t bits_for(uint32_t n) {
  uint32_t bits = 0;
  while (bits < 32u && (1ull << bits) < n) ++bits;
  return bits;
}

// Pairs a step may hold: below 2^30, so 32-bit pair positions, digit starts and scanned
// offsets never wrap (48 GB of per-pair gradients at the limit).
constexpr uint64_t kMaxPairs = (1ull << 30) - 1ull;

}  // namespace

namespace gsk {
void set_last_error(const std::string& message) { g_last_error = message; }
}  // namespace gsk

struct gs_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  // Host targets are uploaded on copy_stream while the step's projection and sort run;
  // the step waits for targets_ready just before the forward raster, the first pass that
  // reads them.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t targets_ready = nullptr;
  // Host targets of the views set last, uploaded by the next step (after its step table,
  // so the table does not queue behind them on the copy engine), once per gs_set_views.
  struct PendingTarget {
    uint32_t offset;
    const uint8_t* host;
    size_t bytes;
  };
  std::vector<PendingTarget> pending_targets;
  bool targets_uploaded = true;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t marks[7] = {};  // pass boundaries, recorded by every step (event nodes inside a captured graph)
  bool profile = false;
  bool count = false;                // GS_STEP_COUNT: the forward counts its blending evaluations
  uint64_t last_contributions = 0;   // their total in the latest counting step
  gsk::Model model;
  gs_tuning tuning{};
  int sm_count = 148;
  // views of the step: host copies, and the step table uploaded each step
  uint32_t n_views = 0;
  std::vector<gs_frame_data> frames;
  gsk::ViewTable vt{};
  uint32_t total_tiles = 0, total_pixels = 0;
  bool has_target = false;
  gsk::StepTable* d_table = nullptr;
  gsk::StepTable* h_table = nullptr;  // pinned
  uint32_t* d_queue = nullptr;        // work-queue counters
  // targets kept in HBM across steps (gs_dataset_set)
  uint32_t* d_dataset = nullptr;
  std::vector<size_t> ds_offset;
  std::vector<uint32_t> ds_width, ds_height;
  // the step captured as a CUDA graph
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<uint64_t> graph_key;
  int graph_launches = 0;
  // (view, slot) buffers
  uint32_t vb_views = 0;
  gsk::ViewBuffers vb;
  uint32_t *dkeys = nullptr, *dvals = nullptr, *dkeys_alt = nullptr, *dvals_alt = nullptr;
  uint32_t* sorted_offsets = nullptr;
  const uint32_t* depth_sorted_keys = nullptr;
  const uint32_t* depth_sorted_vals = nullptr;
  // pixels and tiles
  size_t pixel_cap = 0, tile_cap = 0;
  uint32_t* target = nullptr;
  float4 *pixel_grad = nullptr, *pixel_out = nullptr, *ssim_maps = nullptr;
  float* ssim_last = nullptr;
  uint32_t *pixel_count = nullptr, *image = nullptr;
  float* pixel_dot = nullptr;
  uint2* ranges = nullptr;
  float* tile_loss = nullptr;
  uint32_t* tile_count = nullptr;
  float* tile_part = nullptr;
  uint32_t* tile_done = nullptr;
  // pairs
  uint64_t pair_cap = 0;
  uint32_t *keys = nullptr, *values = nullptr, *keys_alt = nullptr, *values_alt = nullptr, *pair_gaussian = nullptr;
  uint32_t* sorted_g = nullptr;  // each sorted pair's gaussian, in render order (gathered by the ranges pass)
  bool payload_gaussian = false;  // the latest step sorted each pair's gaussian instead of its pre-sort index
  bool graph_payload = false;     // payload_gaussian of the captured graph's steps
  float4* pair_grads = nullptr;
  const uint32_t* sorted_keys = nullptr;
  const uint32_t* sorted_values = nullptr;
  // Step scalars: [0] pairs, [1] emit mismatches (accumulate), [2] and [3] unused,
  // [4 + v] first pair of view v, [4 + kMaxViews + v] its end.
  static constexpr uint32_t kScalars = 4 + 2 * GS_MAX_VIEWS;
  uint32_t* d_scalars = nullptr;
  uint32_t* h_scalars = nullptr;  // pinned
  // Per view: [0..15] the tile sums (losses, then the exposure fit), [16..21] the pose
  // gradient, [22..23] unused.
  static constexpr uint32_t kViewSums = 24;
  double* d_view_sums = nullptr;
  double* h_view_sums = nullptr;  // pinned
  float* pose_partial = nullptr;  // per view and 128 slots: the pose gradient's partial sums
  // Subject motion: the nodes at rest, each slot's binding, the node motions per view (a
  // pinned host copy the setters fill, uploaded with the step), the gradient's per-block
  // partial sums and its totals per view and node.
  uint32_t motion_nodes = 0;
  float4* motion_rest = nullptr;  // kMaxMotionNodes
  uint4* motion_bind = nullptr;   // 2 per slot
  uint32_t motion_bind_cap = 0;
  gsk::MotionNode* d_motion_views = nullptr;  // GS_MAX_VIEWS x kMaxMotionNodes
  gsk::MotionNode* h_motion_views = nullptr;  // pinned
  float* motion_partial = nullptr;
  size_t motion_partial_floats = 0;
  double* d_motion_grad = nullptr;  // GS_MAX_VIEWS x kMaxMotionNodes x 8
  double* h_motion_grad = nullptr;  // pinned
  bool motion_grad_ready = false;
  gsk::SortScratch sort;
  gsk::DensifyScratch dens;
  uint64_t max_pairs_seen = 0;
  uint64_t last_pairs = 0;
  uint32_t densify_slots = 0;  // slots the latest densify marked (the spawn mask's length)
  bool stepped = false;
  int launches = 0;

  ~gs_context() { release(); }

  void release() {
    cudaSetDevice(device);
    for (float4** p : {&model.P, &model.M, &model.V, &model.stats, &vb.splat, &vb.foot, &vb.grad2d, &vb.dir_grad, &pixel_grad,
                       &pixel_out, &ssim_maps, &pair_grads})
      dev_free(*p);
    for (float** p : {&model.SH, &model.MSH, &model.VSH, &pixel_dot, &tile_loss, &tile_part, &pose_partial,
                      &motion_partial, &ssim_last})
      dev_free(*p);
    dev_free(vb.spans);
    dev_free(motion_rest);
    dev_free(motion_bind);
    dev_free(d_motion_views);
    dev_free(d_motion_grad);
    if (h_motion_views) cudaFreeHost(h_motion_views);
    if (h_motion_grad) cudaFreeHost(h_motion_grad);
    h_motion_views = nullptr;
    h_motion_grad = nullptr;
    for (uint32_t** p : {&vb.tiles, &vb.offsets, &dkeys, &dvals, &dkeys_alt, &dvals_alt, &sorted_offsets, &target,
                         &pixel_count, &image, &tile_count, &tile_done, &keys, &values, &keys_alt, &values_alt, &pair_gaussian,
                         &sorted_g,
                         &d_scalars, &sort.hist, &sort.tile_counts, &dens.spawn,
                         &dens.release, &dens.wants, &dens.free_pos, &dens.spawn_pos, &dens.free_list,
                         &dens.counters})
      dev_free(*p);
    dev_free(ranges);
    dev_free(d_table);
    dev_free(d_queue);
    dev_free(d_dataset);
    dev_free(d_view_sums);
    dev_free(sort.scan_lookback);
    drop_graph();
    if (h_table) cudaFreeHost(h_table);
    if (h_scalars) cudaFreeHost(h_scalars);
    if (h_view_sums) cudaFreeHost(h_view_sums);
    h_table = nullptr;
    h_scalars = nullptr;
    h_view_sums = nullptr;
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (cudaEvent_t& e : marks) {
      if (e) cudaEventDestroy(e);
      e = nullptr;
    }
    if (targets_ready) cudaEventDestroy(targets_ready);
    targets_ready = nullptr;
    if (copy_stream) cudaStreamDestroy(copy_stream);
    copy_stream = nullptr;
    if (stream) cudaStreamDestroy(stream);
    ev0 = ev1 = nullptr;
    stream = nullptr;
  }

  void drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
    graph_key.clear();
  }

  void check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(GS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }

  // (view, slot) buffers for `views` views of `cap` slots.
  void reserve_views(uint32_t views) {
    if (views <= vb_views) return;
    drop_graph();
    const size_t n = size_t(views) * model.cap;
    dev_alloc(vb.splat, n * 3);
    dev_alloc(vb.foot, n);
    dev_alloc(vb.spans, n);
    dev_alloc(vb.tiles, n);
    dev_alloc(vb.offsets, n);
    dev_alloc(vb.grad2d, n * 3);
    dev_alloc(vb.dir_grad, model.cap);
    dev_alloc(dkeys, n);
    dev_alloc(dvals, n);
    dev_alloc(dkeys_alt, n);
    dev_alloc(dvals_alt, n);
    dev_alloc(sorted_offsets, n);
    dev_alloc(pose_partial, size_t(views) * gsk::pose_blocks(model.cap) * 8u);
    GS_CUDA_TRY(cudaMemsetAsync(vb.tiles, 0, n * sizeof(uint32_t), stream));
    const uint32_t sort_tiles = uint32_t((n + gsk::kSortTile - 1) / gsk::kSortTile);
    if (sort_tiles > sort.count_tiles) {
      dev_alloc(sort.tile_counts, size_t(sort_tiles) * 256);
      sort.count_tiles = sort_tiles;
    }
    const uint32_t scan_tiles = uint32_t((n + gsk::kScanTile - 1) / gsk::kScanTile);
    if (scan_tiles > sort.scan_tiles) {
      dev_alloc(sort.scan_lookback, scan_tiles);
      sort.scan_tiles = scan_tiles;
    }
    vb_views = views;
  }

  void reserve_pixels(size_t pixels, size_t tiles) {
    if (pixels > pixel_cap || tiles + 1 > tile_cap) drop_graph();
    if (pixels > pixel_cap) {
      dev_alloc(target, pixels);
      dev_alloc(pixel_grad, pixels);
      dev_alloc(pixel_out, pixels);
      dev_alloc(ssim_maps, pixels * 2);
      dev_alloc(ssim_last, pixels);
      dev_alloc(pixel_count, pixels);
      dev_alloc(image, pixels);
      dev_alloc(pixel_dot, pixels);
      pixel_cap = pixels;
    }
    if (tiles + 1 > tile_cap) {
      dev_alloc(ranges, tiles + 1);
      dev_alloc(tile_loss, (tiles + 1) * 16);
      dev_alloc(tile_count, tiles + 1);
      dev_alloc(tile_part, (tiles + 1) * gsk::kTileWarpSlots * 16);
      dev_alloc(tile_done, tiles + 1);
      GS_CUDA_TRY(cudaMemsetAsync(tile_done, 0, (tiles + 1) * sizeof(uint32_t), stream));  // then each tile resets its own
      tile_cap = tiles + 1;
    }
  }

  void reserve_pairs(uint64_t expected) {
    const uint64_t wanted = expected + expected / 8;
    if (wanted <= pair_cap && pair_cap > 0) return;
    if (expected > kMaxPairs) fail(GS_ERR_CAPACITY, "more tile-gaussian pairs than the pair buffers can hold (" +
                                                        std::to_string(expected) + ")");
    const uint64_t n = std::min<uint64_t>(kMaxPairs, std::max<uint64_t>(wanted + wanted / 4, tuning.min_pair_capacity));
    drop_graph();
    dev_alloc(keys, n);
    dev_alloc(values, n);
    dev_alloc(keys_alt, n);
    dev_alloc(values_alt, n);
    dev_alloc(pair_gaussian, n);
    dev_alloc(sorted_g, n);
    dev_alloc(pair_grads, n * 3);
    const uint32_t sort_tiles = uint32_t((n + gsk::kSortTile - 1) / gsk::kSortTile);
    if (sort_tiles > sort.count_tiles) {
      dev_alloc(sort.tile_counts, size_t(sort_tiles) * 256);
      sort.count_tiles = sort_tiles;
    }
    pair_cap = n;
  }

  // Milliseconds between two recorded events (0 if they cannot be timed).
  static float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
      (void)cudaGetLastError();
      ms = 0.0f;
    }
    return ms;
  }

  // Inside a stream capture a plain record only orders the capture's streams; an external
  // record becomes an event node that each replay records, so the marks time replays too.
  void mark(int k) {
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    GS_CUDA_TRY(cudaStreamIsCapturing(stream, &capture));
    GS_CUDA_TRY(cudaEventRecordWithFlags(
        marks[k], stream, capture == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault));
  }

  // Everything one step puts on the stream: the step table upload, the queue reset, the
  // launch sequence and the readback of the pair count and loss sums.
  // The step table is uploaded by run_step before this (outside any graph).
  void enqueue_step(bool train, uint32_t degree) {
    GS_CUDA_TRY(cudaMemsetAsync(d_queue, 0, sizeof(uint32_t) * gsk::kQueueCount, stream));
    record(train, degree);
    GS_CUDA_TRY(cudaMemcpyAsync(h_scalars, d_scalars, kScalars * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    GS_CUDA_TRY(cudaMemcpyAsync(h_view_sums, d_view_sums, sizeof(double) * kViewSums * n_views,
                                cudaMemcpyDeviceToHost, stream));
    if (train && (motion_mode() & 2u))
      GS_CUDA_TRY(cudaMemcpyAsync(h_motion_grad, d_motion_grad, sizeof(double) * 8 * gsk::kMaxMotionNodes * n_views,
                                  cudaMemcpyDeviceToHost, stream));
  }

  // The step as a CUDA graph: captured once per launch structure (views, slots, buffer
  // sizes, SH degree, mode, tuning), replayed while only the step table changes.
  void launch_graph(bool train, uint32_t degree) {
    const bool ssim = (frames[0].model[3] & GS_FLAG_SSIM) != 0u && has_target;
    const std::vector<uint64_t> key = {n_views, model.slots, model.cap, pair_cap, tile_cap, pixel_cap, degree,
                                       train ? 1u : 0u, ssim ? 1u : 0u, tuning.deterministic,
                                       tuning.forward_pixels, tuning.backward_pixels, tuning.backward_batch,
                                       tuning.sort_digit_bits, pose_mode(), motion_mode(), motion_nodes};
    if (graph_exec == nullptr || key != graph_key) {
      drop_graph();
      cudaGraph_t g = nullptr;
      GS_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      launches = 0;
      try {
        enqueue_step(train, degree);
      } catch (...) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      GS_CUDA_TRY(cudaStreamEndCapture(stream, &g));
      const cudaError_t e = cudaGraphInstantiate(&graph_exec, g, 0);
      cudaGraphDestroy(g);
      GS_CUDA_TRY(e);
      graph_key = key;
      graph_launches = launches;
      graph_payload = payload_gaussian;
    }
    launches = graph_launches;
    payload_gaussian = graph_payload;  // a step recorded since (without the graph) may have changed it
    GS_CUDA_TRY(cudaGraphLaunch(graph_exec, stream));
  }

  void run_step(bool train, gs_step_result* out, bool allow_graph = true) {
    if (n_views == 0) fail(GS_ERR_INVALID, "gs_step: no views (gs_set_views first)");
    if (train && !has_target) fail(GS_ERR_INVALID, "gs_step: training needs target images");
    const uint32_t degree = frames[0].model[1];
    uint32_t retries = 0;
    for (;;) {
      const uint64_t guess = max_pairs_seen > 0 ? max_pairs_seen
                             : tuning.initial_pairs ? tuning.initial_pairs
                                                    : uint64_t(model.slots) * 4u * n_views;
      reserve_pairs(guess);
      h_table->vt = vt;
      for (uint32_t v = 0; v < n_views; ++v) {
        gs_frame_data& f = h_table->frames[v];
        f = frames[v];
        f.model[0] = model.slots;
        f.model[2] = model.sh_stride;
        f.limits[0] = uint32_t(pair_cap);
        f.limits[3] = uint32_t(pair_cap);
      }
      // The table first, then the targets of a new view set on the copy stream (the step
      // waits for them before the forward raster; views without host targets record an
      // event that is already complete).
      GS_CUDA_TRY(cudaMemcpyAsync(d_table, h_table, sizeof(gsk::StepTable), cudaMemcpyHostToDevice, stream));
      const uint32_t motion = motion_mode();
      if (motion != 0u) {
        GS_CUDA_TRY(cudaMemcpyAsync(d_motion_views, h_motion_views,
                                    sizeof(gsk::MotionNode) * gsk::kMaxMotionNodes * n_views, cudaMemcpyHostToDevice,
                                    stream));
        if (train && (motion & 2u)) reserve_motion_partial();
      }
      if (!targets_uploaded) {
        for (const PendingTarget& p : pending_targets)
          GS_CUDA_TRY(cudaMemcpyAsync(target + p.offset, p.host, p.bytes, cudaMemcpyHostToDevice, copy_stream));
        GS_CUDA_TRY(cudaEventRecord(targets_ready, copy_stream));
        targets_uploaded = true;
      }
      GS_CUDA_TRY(cudaEventRecord(ev0, stream));
      // The pass events are part of the step's launch sequence, so a graph replay records
      // them too and a profiled step can run as a replay.
      if (tuning.graph && allow_graph && !count) {
        launch_graph(train, degree);
      } else {
        launches = 0;
        enqueue_step(train, degree);
      }
      GS_CUDA_TRY(cudaEventRecord(ev1, stream));
      GS_CUDA_TRY(cudaStreamSynchronize(stream));
      check_launch("step");
      const uint64_t pairs = h_scalars[0];
      if (count) last_contributions = uint64_t(h_scalars[2]) | uint64_t(h_scalars[3]) << 32;
      last_pairs = pairs;
      max_pairs_seen = std::max(max_pairs_seen, pairs);
      stepped = true;
      const bool overflow = pairs > pair_cap;
      if (overflow && tuning.retry && retries < 4) {
        ++retries;
        continue;  // the step left the model alone; grow and run it again
      }
      if (out) {
        std::memset(out, 0, sizeof(*out));
        out->n_views = n_views;
        out->overflow = overflow ? 1u : 0u;
        out->retries = retries;
        out->tile_mismatch = h_scalars[1];
        view_pairs(out->pairs);
        for (uint32_t v = 0; v < n_views; ++v) {
          const double* s = h_view_sums + size_t(v) * kViewSums;
          for (int k = 0; k < 8; ++k) out->losses[v][k] = s[k];
          for (int k = 0; k < 8; ++k) out->fit[v][k] = s[8 + k];
          if (train && (pose_mode() & 1u))
            for (int k = 0; k < 6; ++k) out->pose_grad[v][k] = s[16 + k];
        }
        out->gpu_ms = elapsed(ev0, ev1);
        motion_grad_ready = train && (motion_mode() & 2u) != 0u;
        out->kernels = uint32_t(launches);
        if (profile)
          for (int k = 0; k < 6; ++k) out->pass_ms[k] = (train || k < 4) ? elapsed(marks[k], marks[k + 1]) : 0.0f;
      }
      return;
    }
  }

  // Mean device time of `steps` training steps under tuning `t`, after one untimed step
  // (graph capture, buffer growth).
  float time_tuning(const gs_tuning& t, uint32_t steps) {
    tuning = t;
    drop_graph();
    run_step(true, nullptr);
    float ms = 0.0f;
    for (uint32_t k = 0; k < steps; ++k) {
      gs_step_result r;
      run_step(true, &r);
      ms += r.gpu_ms;
    }
    return ms / float(steps);
  }

  // gs_autotune: greedy over the knobs, the model restored afterwards (trainer.cpp:876-897
  // times its backward variants on training steps the same way and keeps the fastest).
  void autotune(uint32_t steps) {
    if (n_views == 0 || !has_target) fail(GS_ERR_INVALID, "gs_autotune: needs views with targets (gs_set_views)");
    const size_t planes4 = sizeof(float4) * model.cap, planes_sh = sizeof(float) * size_t(model.sh_stride) * model.cap;
    struct Part {
      void* ptr;
      size_t bytes;
    };
    const Part parts[] = {{model.P, 4 * planes4},     {model.M, 4 * planes4},      {model.V, 4 * planes4},
                          {model.stats, planes4},     {model.SH, planes_sh},       {model.MSH, planes_sh},
                          {model.VSH, planes_sh}};
    size_t total = 0;
    for (const Part& p : parts) total += p.bytes;
    uint8_t* backup = nullptr;
    if (cudaMalloc(&backup, total) != cudaSuccess) {
      cudaGetLastError();
      fail(GS_ERR_NO_MEMORY, "gs_autotune: no device memory for a copy of the model");
    }
    size_t at = 0;
    for (const Part& p : parts) {
      if (p.bytes) cudaMemcpyAsync(backup + at, p.ptr, p.bytes, cudaMemcpyDeviceToDevice, stream);
      at += p.bytes;
    }
    const gs_tuning start = tuning;
    gs_tuning best = start;
    std::string failure;
    int failure_code = GS_OK;
    try {
      float best_ms = time_tuning(best, steps);
      auto consider = [&](gs_tuning t) {
        const float ms = time_tuning(t, steps);
        if (ms < best_ms) {
          best_ms = ms;
          best = t;
        }
      };
      if (start.tune_reduction) {  // fixed-order sums or atomics, then the rest under the faster
        gs_tuning t = best;
        t.deterministic = best.deterministic ? 0u : 1u;
        consider(t);
      }
      const uint32_t fpx0 = best.forward_pixels;
      for (uint32_t fpx : {1u, 2u, 4u})
        if (fpx != fpx0) {
          gs_tuning t = best;
          t.forward_pixels = fpx;
          consider(t);
        }
      if (best.stage_async) {  // the forward's round size (only its block kernel stages rounds of it)
        gs_tuning t = best;
        t.forward_batch = best.forward_batch == 128u ? 256u : 128u;
        consider(t);
      }
      const uint32_t bpx0 = best.backward_pixels, batch0 = best.backward_batch;
      // (The fast backward stages 32 splats per warp whatever backward_batch says, so in
      // fast mode only the pixels per thread are tried.)
      for (uint32_t bpx : {2u, 4u})
        for (uint32_t batch : {32u, 64u})
          if ((bpx != bpx0 || batch != batch0) && (best.deterministic || batch == batch0)) {
            gs_tuning t = best;
            t.backward_pixels = bpx;
            t.backward_batch = batch;
            consider(t);
          }
      if (bpx0 != 8u) {  // one warp per tile (its rounds are 32 splats whatever backward_batch says)
        gs_tuning t = best;
        t.backward_pixels = 8u;
        consider(t);
      }
      const uint32_t digits0 = best.sort_digit_bits;
      for (uint32_t digits : {6u, 7u, 8u})
        if (digits != digits0) {
          gs_tuning t = best;
          t.sort_digit_bits = digits;
          consider(t);
        }
    } catch (const Failure& e) {
      failure_code = e.code;
      failure = e.message;
    }
    at = 0;
    for (const Part& p : parts) {
      if (p.bytes) cudaMemcpyAsync(p.ptr, backup + at, p.bytes, cudaMemcpyDeviceToDevice, stream);
      at += p.bytes;
    }
    const cudaError_t e = cudaStreamSynchronize(stream);
    cudaFree(backup);
    tuning = failure_code == GS_OK ? best : start;
    drop_graph();
    if (failure_code != GS_OK) fail(failure_code, "gs_autotune: " + failure);
    if (e != cudaSuccess) fail(GS_ERR_CUDA, std::string("gs_autotune: ") + cudaGetErrorString(e));
  }

  // Pairs of each view: pairs are ordered by view, so the first pair of view v+1 bounds v.
  void view_pairs(uint64_t* out) {
    if (n_views == 1) {
      out[0] = last_pairs;
      return;
    }
    // The views' spans in the sorted pairs, found by k_ranges (stored pairs only).
    for (uint32_t v = 0; v < n_views; ++v) {
      const uint32_t lo = h_scalars[4 + v], hi = h_scalars[4 + GS_MAX_VIEWS + v];
      out[v] = hi > lo ? hi - lo : 0;
    }
  }

  gsk::StepPointers step_pointers() const {
    gsk::StepPointers sp;
    sp.frames = d_table->frames;
    sp.vt = &d_table->vt;
    sp.n_views = n_views;
    sp.tile_cap = tile_cap > 0 ? uint32_t(tile_cap - 1) : 0u;
    sp.queue = d_queue;
    sp.sm_count = sm_count;
    return sp;
  }

  gsk::RasterBuffers raster_buffers() const {
    gsk::RasterBuffers rb;
    rb.ranges = ranges;
    rb.values = sorted_values;
    rb.gauss = payload_gaussian ? sorted_values : sorted_g;
    rb.pixel_grad = pixel_grad;
    rb.pixel_out = pixel_out;
    rb.pixel_count = pixel_count;
    rb.image = image;
    rb.pixel_dot = pixel_dot;
    rb.tile_loss = tile_loss;
    rb.tile_count = tile_count;
    rb.tile_part = tile_part;
    rb.tile_done = tile_done;
    rb.ssim_maps = ssim_maps;
    rb.ssim_last = ssim_last;
    return rb;
  }

  // Bit 0: some view moves with the subject; bit 1: some view asks for its motion gradient.
  uint32_t motion_mode() const {
    if (motion_nodes == 0u) return 0u;
    uint32_t m = 0u;
    for (uint32_t v = 0; v < n_views; ++v) {
      if (frames[v].model[3] & GS_FLAG_MOTION) m |= 1u;
      if (frames[v].model[3] & GS_FLAG_MOTION_GRAD) m |= 2u;
    }
    return m;
  }

  gsk::Motion motion_state() const {
    gsk::Motion m;
    m.nodes = motion_nodes;
    m.rest = motion_rest;
    m.bind = motion_bind;
    m.views = d_motion_views;
    return m;
  }

  void reserve_motion_partial() {
    const size_t wanted =
        size_t(n_views) * gsk::motion_blocks(model.slots, sm_count) * gsk::kMaxMotionNodes * 8u;
    if (wanted <= motion_partial_floats) return;
    drop_graph();
    dev_alloc(motion_partial, wanted);
    motion_partial_floats = wanted;
  }

  void bind_motion() {
    if (motion_nodes == 0u || model.slots == 0u) return;
    gsk::launch_motion_bind(model, motion_state(), stream);
    GS_CUDA_TRY(cudaStreamSynchronize(stream));
    check_launch("motion bind");
  }

  // Bit 0: some view asks for its pose gradient; bit 1: the step changes nothing (the
  // first view's GS_FLAG_POSE_ONLY).
  uint32_t pose_mode() const {
    uint32_t m = 0u;
    for (uint32_t v = 0; v < n_views; ++v)
      if (frames[v].model[3] & GS_FLAG_POSE_GRAD) m |= 1u;
    if (n_views > 0 && (frames[0].model[3] & GS_FLAG_POSE_ONLY)) m |= 2u;
    return m;
  }

  // The launch sequence of one step (trainer.cpp:825-831), all on `stream`.
  void record(bool train, uint32_t degree) {
    const gsk::StepPointers sp = step_pointers();
    const uint32_t items = n_views * model.slots;
    const bool det = tuning.deterministic != 0u;
    // An atomic training step needs no pre-sort pair index: the sort carries each pair's
    // gaussian, which the raster passes stage from directly (no gather). Deterministic and
    // forward-only steps keep the index (per-pair gradients, the render-order snapshots).
    payload_gaussian = train && !det;
    vb.view_word = train && !det;  // the projection zeroes grad2d for the atomics and leaves the view word
    GS_CUDA_TRY(cudaMemsetAsync(d_scalars, 0, sizeof(uint32_t), stream));  // [0] pairs; [1] mismatches accumulate
    const uint32_t motion = motion_mode();
    const gsk::Motion mo = motion_state();
    const gsk::Motion* moving = (motion & 1u) ? &mo : nullptr;
    mark(0);
    gsk::launch_project(sp, model, degree, vb, dkeys, dvals, train && !det, moving, stream);
    launches += model.slots ? 1 : 0;
    mark(1);
    // Depth sort of every (view, slot): key = view << 16 | depth16.
    const int depth_bits = 16 + int(bits_for(n_views));
    const int digit_bits = tuning.sort_digit_bits ? int(tuning.sort_digit_bits) : 8;
    const bool in_alt = gsk::radix_sort_pairs(sort, dkeys, dvals, dkeys_alt, dvals_alt, nullptr, items, depth_bits,
                                              stream, &launches, digit_bits);
    depth_sorted_keys = in_alt ? dkeys_alt : dkeys;
    depth_sorted_vals = in_alt ? dvals_alt : dvals;
    // Offsets of each item's pairs in depth order; the total is the step's pair count.
    gsk::exclusive_scan(sort, vb.tiles, depth_sorted_vals, sorted_offsets, items, d_scalars, stream, &launches);
    // With the gaussian as the payload nothing reads the per-pair gaussian: not written.
    gsk::launch_emit(sp, vb, model.cap, items, depth_sorted_vals, sorted_offsets, d_scalars, uint32_t(pair_cap), keys,
                     values, payload_gaussian ? nullptr : pair_gaussian, pair_grads, d_scalars + 1, payload_gaussian,
                     stream);
    launches += items ? 1 : 0;
    const uint32_t max_tiles = uint32_t(tile_cap - 1);
    const int tile_bits = int(bits_for(max_tiles + 1));
    const bool pairs_alt = gsk::radix_sort_pairs(sort, keys, values, keys_alt, values_alt, d_scalars,
                                                 uint32_t(pair_cap), std::max(tile_bits, 1), stream, &launches,
                                                 digit_bits);
    sorted_keys = pairs_alt ? keys_alt : keys;
    sorted_values = pairs_alt ? values_alt : values;
    GS_CUDA_TRY(cudaMemsetAsync(ranges, 0, sizeof(uint2) * (max_tiles + 1), stream));
    GS_CUDA_TRY(cudaMemsetAsync(d_scalars + 4, 0, 2 * GS_MAX_VIEWS * sizeof(uint32_t), stream));
    const gsk::PairGather gather{sorted_values, pair_gaussian, sorted_g};
    gsk::launch_ranges(sorted_keys, d_scalars, uint32_t(pair_cap), ranges, sp.vt, d_scalars + 4,
                       payload_gaussian ? nullptr : &gather, stream);
    ++launches;
    mark(2);
    const gsk::RasterBuffers rb = raster_buffers();
    {
      cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
      GS_CUDA_TRY(cudaStreamIsCapturing(stream, &capture));
      GS_CUDA_TRY(cudaStreamWaitEvent(stream, targets_ready,
                                      capture == cudaStreamCaptureStatusActive ? cudaEventWaitExternal : 0u));
    }
    unsigned long long* contributions = nullptr;
    if (count) {  // d_scalars[2..3]: a 64-bit counter
      contributions = reinterpret_cast<unsigned long long*>(d_scalars + 2);
      GS_CUDA_TRY(cudaMemsetAsync(contributions, 0, sizeof(unsigned long long), stream));
    }
    gsk::launch_raster_forward(sp, vb, rb, tuning.forward_pixels ? int(tuning.forward_pixels) : 2,
                               tuning.forward_batch ? int(tuning.forward_batch) : 256, tuning.stage_async != 0u,
                               contributions, stream);
    ++launches;
    mark(3);
    const bool ssim = (frames[0].model[3] & GS_FLAG_SSIM) != 0u && has_target;
    if (ssim) {
      gsk::launch_ssim(sp, rb, stream);
      ++launches;
      if (train) {
        gsk::launch_ssim_grad(sp, rb, stream);
        ++launches;
      }
    }
    gsk::launch_loss_reduce(sp, tile_loss, d_view_sums, kViewSums, d_view_sums + kViewSums * GS_MAX_VIEWS, stream);
    launches += 2;
    mark(4);
    if (train) {
      const int px = tuning.backward_pixels ? int(tuning.backward_pixels) : 4;
      const int batch = tuning.backward_batch ? int(tuning.backward_batch) : 64;
      gsk::launch_raster_backward(sp, vb, rb, pair_grads, det, px, batch, tuning.stage_async != 0u, d_scalars,
                                  uint32_t(pair_cap), stream);
      ++launches;
      mark(5);
      if (det) {
        gsk::launch_pair_sum(vb, items, depth_sorted_vals, sorted_offsets, pair_grads, d_scalars, uint32_t(pair_cap),
                             stream);
        ++launches;
      }
      const uint32_t pose = pose_mode();
      if (pose & 1u) {
        gsk::launch_pose_grad(sp, model, degree, vb, d_scalars, uint32_t(pair_cap), moving, pose_partial,
                              d_view_sums + 16, kViewSums, stream);
        launches += model.slots ? 2 : 1;
      }
      if (motion & 2u) {
        gsk::launch_motion_grad(sp, model, degree, vb, d_scalars, uint32_t(pair_cap), mo, motion_partial,
                                d_motion_grad, stream);
        launches += model.slots ? 2 : 1;
      }
      if ((pose & 2u) == 0u) {
        gsk::launch_step(sp, model, degree, vb, d_scalars, uint32_t(pair_cap), moving, stream);
        launches += model.slots ? (degree > 0 ? 2 : 1) : 0;
      }
      mark(6);
    }
    check_launch("launch");
  }

  // The views of the next step. Targets come from host images (copied into the step's
  // target buffer) or from images already in HBM (`images`: dataset indices), or neither.
  void set_views(uint32_t n, const gs_frame_data* fr, const uint8_t* const* targets, const uint32_t* images) {
    if (n == 0 || n > GS_MAX_VIEWS) fail(GS_ERR_INVALID, "gs_set_views: 1 to 16 views");
    if (model.cap == 0) fail(GS_ERR_INVALID, "gs_set_views: no model (gs_model_init first)");
    std::vector<gs_frame_data> next(fr, fr + n);
    gsk::ViewTable t{};
    t.n_views = n;
    uint64_t tiles = 0, pixels = 0;
    for (uint32_t v = 0; v < n; ++v) {
      gs_frame_data& f = next[v];
      const uint32_t w = f.image[0], h = f.image[1];
      if (w == 0 || h == 0) fail(GS_ERR_INVALID, "gs_set_views: empty image");
      f.image[2] = (w + gsk::kTile - 1) / gsk::kTile;
      f.image[3] = (h + gsk::kTile - 1) / gsk::kTile;
      if (f.model[1] > 3u || gsk::sh_rest_coeffs(f.model[1]) * 3u > model.sh_stride)
        fail(GS_ERR_INVALID, "gs_set_views: active SH degree beyond the model's SH storage");
      if (v > 0 && f.model[1] != next[0].model[1])
        fail(GS_ERR_INVALID, "gs_set_views: the views of a step share the active SH degree");
      if (images != nullptr) {
        if (images[v] >= ds_width.size()) fail(GS_ERR_INVALID, "gs_set_views_dataset: no such image");
        if (ds_width[images[v]] != w || ds_height[images[v]] != h)
          fail(GS_ERR_INVALID, "gs_set_views_dataset: image size differs from the view's");
      }
      t.tile_base[v] = uint32_t(tiles);
      t.pixel_base[v] = uint32_t(pixels);
      tiles += uint64_t(f.image[2]) * f.image[3];
      pixels += uint64_t(w) * h;
    }
    if (tiles >= (1ull << 24) || pixels >= (1ull << 31)) fail(GS_ERR_INVALID, "gs_set_views: images too large");
    for (uint32_t v = n; v <= GS_MAX_VIEWS; ++v) {
      t.tile_base[v] = uint32_t(tiles);
      t.pixel_base[v] = uint32_t(pixels);
    }
    t.total_tiles = uint32_t(tiles);
    t.total_pixels = uint32_t(pixels);
    if (targets != nullptr)
      for (uint32_t v = 0; v < n; ++v)
        if (targets[v] == nullptr) fail(GS_ERR_INVALID, "gs_set_views: missing target image");
    std::vector<PendingTarget> pending;
    reserve_views(n);
    reserve_pixels(pixels, tiles);
    for (uint32_t v = 0; v < n; ++v) {
      if (targets != nullptr) {
        t.target[v] = target + t.pixel_base[v];
        const size_t bytes = size_t(next[v].image[0]) * next[v].image[1] * 4;
        pending.push_back({t.pixel_base[v], targets[v], bytes});
      } else if (images != nullptr) {
        t.target[v] = d_dataset + ds_offset[images[v]];
      }
    }
    frames = std::move(next);
    vt = t;
    n_views = n;
    total_tiles = t.total_tiles;
    total_pixels = t.total_pixels;
    pending_targets = std::move(pending);
    targets_uploaded = false;
    has_target = targets != nullptr || images != nullptr;
  }

  void set_dataset(uint32_t n, const uint32_t* widths, const uint32_t* heights, const uint8_t* const* rgba) {
    size_t total = 0;
    for (uint32_t i = 0; i < n; ++i) {
      if (widths[i] == 0 || heights[i] == 0 || rgba[i] == nullptr) fail(GS_ERR_INVALID, "gs_dataset_set: empty image");
      total += size_t(widths[i]) * heights[i];
    }
    GS_CUDA_TRY(cudaStreamSynchronize(stream));
    drop_graph();
    ds_offset.assign(n, 0);
    ds_width.assign(widths, widths + n);
    ds_height.assign(heights, heights + n);
    dev_alloc(d_dataset, total);
    size_t off = 0;
    for (uint32_t i = 0; i < n; ++i) {
      ds_offset[i] = off;
      GS_CUDA_TRY(cudaMemcpyAsync(d_dataset + off, rgba[i], size_t(widths[i]) * heights[i] * 4,
                                  cudaMemcpyHostToDevice, stream));
      off += size_t(widths[i]) * heights[i];
    }
    GS_CUDA_TRY(cudaStreamSynchronize(stream));
    // Views that pointed at the old dataset must be set again.
    if (has_target && n_views > 0) n_views = 0;
  }
};

namespace gsk {
namespace {

__global__ void k_params_to_planes(const float* __restrict__ params16, const float* __restrict__ sh, uint32_t count,
                                   uint32_t cap, uint32_t stride, float4* P, float* SH) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float4* p = reinterpret_cast<const float4*>(params16) + size_t(i) * 4u;
#pragma unroll
  for (int k = 0; k < 4; ++k) P[size_t(k) * cap + i] = p[k];
  if (sh != nullptr)
    for (uint32_t k = 0; k < stride; ++k) SH[size_t(k) * cap + i] = sh[size_t(i) * stride + k];
}

__global__ void k_planes_to_params(const float4* P, const float* SH, uint32_t count, uint32_t cap, uint32_t stride,
                                   float* params16, float* sh) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  if (params16 != nullptr) {
    float4* p = reinterpret_cast<float4*>(params16) + size_t(i) * 4u;
#pragma unroll
    for (int k = 0; k < 4; ++k) p[k] = P[size_t(k) * cap + i];
  }
  if (sh != nullptr)
    for (uint32_t k = 0; k < stride; ++k) sh[size_t(i) * stride + k] = SH[size_t(k) * cap + i];
}

__global__ void k_projected_record(const float4* splat, const float4* foot, uint32_t base, uint32_t slots,
                                   float4* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= slots) return;
  const size_t g = size_t(base) + i;
  out[size_t(i) * 4u] = splat[g * 3u];
  out[size_t(i) * 4u + 1u] = splat[g * 3u + 1u];
  out[size_t(i) * 4u + 2u] = splat[g * 3u + 2u];
  out[size_t(i) * 4u + 3u] = foot[g];
}

}  // namespace

void launch_params_to_planes(const float* params16, const float* sh, uint32_t count, const Model& m, cudaStream_t st) {
  if (count == 0) return;
  k_params_to_planes<<<(count + 255u) / 256u, 256, 0, st>>>(params16, sh, count, m.cap, m.sh_stride, m.P, m.SH);
}

void launch_planes_to_params(const Model& m, const float4* P, const float* SH, float* params16, float* sh,
                             uint32_t count, cudaStream_t st) {
  if (count == 0) return;
  k_planes_to_params<<<(count + 255u) / 256u, 256, 0, st>>>(P, SH, count, m.cap, m.sh_stride, params16, sh);
}

void launch_projected_record(const ViewBuffers& vb, uint32_t view, uint32_t cap, uint32_t slots, float* out16,
                             cudaStream_t st) {
  if (slots == 0) return;
  k_projected_record<<<(slots + 255u) / 256u, 256, 0, st>>>(vb.splat, vb.foot, view * cap, slots,
                                                            reinterpret_cast<float4*>(out16));
}

}  // namespace gsk

namespace {

// Copies `count` items of a device array to host through a temporary device buffer
// produced by `fill` (layout conversions).
template <typename T, typename F>
void download_via(gs_context* c, size_t count, T* host, F fill) {
  T* tmp = nullptr;
  dev_alloc(tmp, count);
  fill(tmp);
  const cudaError_t e1 = cudaMemcpyAsync(host, tmp, count * sizeof(T), cudaMemcpyDeviceToHost, c->stream);
  const cudaError_t e2 = cudaStreamSynchronize(c->stream);
  dev_free(tmp);
  GS_CUDA_TRY(e1);
  GS_CUDA_TRY(e2);
}

}  // namespace

extern "C" {

const char* gs_last_error(void) { return g_last_error.c_str(); }

int gs_create(int device, gs_context** out) {
  return guarded([&] {
    if (out == nullptr) fail(GS_ERR_INVALID, "gs_create: null output");
    *out = nullptr;
    int count = 0;
    GS_CUDA_TRY(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) fail(GS_ERR_INVALID, "gs_create: no CUDA device " + std::to_string(device));
    cudaDeviceProp prop{};
    GS_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
      fail(GS_ERR_INVALID, std::string("gs_create: libgs_cuda is built for sm_100a; device is ") + prop.name);
    GS_CUDA_TRY(cudaSetDevice(device));
    gs_context* c = new gs_context();
    c->device = device;
    c->tuning.min_pair_capacity = 1u << 16;
    c->tuning.deterministic = 1u;
    c->tuning.forward_pixels = 2u;
    c->tuning.backward_pixels = 4u;
    c->tuning.backward_batch = 64u;
    c->tuning.sort_digit_bits = 8u;
    c->tuning.forward_batch = 256u;
    c->tuning.retry = 1u;
    c->tuning.graph = 0u;
    try {
      GS_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      GS_CUDA_TRY(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
      GS_CUDA_TRY(cudaEventCreateWithFlags(&c->targets_ready, cudaEventDisableTiming));
      GS_CUDA_TRY(cudaEventCreate(&c->ev0));
      GS_CUDA_TRY(cudaEventCreate(&c->ev1));
      for (cudaEvent_t& e : c->marks) GS_CUDA_TRY(cudaEventCreate(&e));
      GS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&c->h_table), sizeof(gsk::StepTable)));
      std::memset(c->h_table, 0, sizeof(gsk::StepTable));
      GS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&c->h_scalars), gs_context::kScalars * sizeof(uint32_t)));
      GS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&c->h_view_sums),
                                 gs_context::kViewSums * sizeof(double) * GS_MAX_VIEWS));
      dev_alloc(c->d_table, 1);
      dev_alloc(c->d_queue, gsk::kQueueCount);
      c->sm_count = prop.multiProcessorCount;
      dev_alloc(c->d_scalars, gs_context::kScalars);
      // The views' sums, then the loss reduction's per-slice scratch.
      dev_alloc(c->d_view_sums, (gs_context::kViewSums + gsk::kLossParts * 16u) * GS_MAX_VIEWS);
      dev_alloc(c->sort.hist, 8 * 256);
      GS_CUDA_TRY(cudaMemset(c->d_scalars, 0, gs_context::kScalars * sizeof(uint32_t)));
    } catch (...) {
      delete c;
      throw;
    }
    *out = c;
  });
}

int gs_destroy(gs_context* ctx) {
  return guarded([&] { delete ctx; });
}

int gs_model_init(gs_context* c, uint32_t capacity, uint32_t sh_stride, const float* params16, const float* sh,
                  uint32_t count) {
  return guarded([&] {
    if (c == nullptr) fail(GS_ERR_INVALID, "gs_model_init: null context");
    if (capacity == 0 || count > capacity) fail(GS_ERR_INVALID, "gs_model_init: count must be within 1..capacity");
    if (sh_stride % 3u != 0u || sh_stride > 45u) fail(GS_ERR_INVALID, "gs_model_init: sh_stride must be 0, 9, 24 or 45");
    if (count > 0 && params16 == nullptr) fail(GS_ERR_INVALID, "gs_model_init: null params");
    if (count > 0 && sh_stride > 0 && sh == nullptr) fail(GS_ERR_INVALID, "gs_model_init: null sh");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    GS_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->drop_graph();
    gsk::Model& m = c->model;
    dev_free(m.P);
    dev_free(m.M);
    dev_free(m.V);
    dev_free(m.stats);
    dev_free(m.SH);
    dev_free(m.MSH);
    dev_free(m.VSH);
    c->vb_views = 0;
    m.cap = capacity;
    m.slots = count;
    m.sh_stride = sh_stride;
    dev_alloc(m.P, size_t(capacity) * 4);
    dev_alloc(m.M, size_t(capacity) * 4);
    dev_alloc(m.V, size_t(capacity) * 4);
    dev_alloc(m.stats, capacity);
    dev_alloc(m.SH, size_t(capacity) * sh_stride);
    dev_alloc(m.MSH, size_t(capacity) * sh_stride);
    dev_alloc(m.VSH, size_t(capacity) * sh_stride);
    for (float4* p : {m.P, m.M, m.V}) GS_CUDA_TRY(cudaMemsetAsync(p, 0, sizeof(float4) * 4 * capacity, c->stream));
    GS_CUDA_TRY(cudaMemsetAsync(m.stats, 0, sizeof(float4) * capacity, c->stream));
    for (float* p : {m.SH, m.MSH, m.VSH})
      GS_CUDA_TRY(cudaMemsetAsync(p, 0, sizeof(float) * std::max<size_t>(1, size_t(capacity) * sh_stride), c->stream));
    dev_alloc(c->dens.spawn, capacity);
    dev_alloc(c->dens.release, capacity);
    dev_alloc(c->dens.wants, capacity);
    dev_alloc(c->dens.free_pos, capacity);
    dev_alloc(c->dens.spawn_pos, capacity);
    dev_alloc(c->dens.free_list, capacity);
    dev_alloc(c->dens.counters, 4);
    const uint32_t scan_tiles = (capacity + gsk::kScanTile - 1) / gsk::kScanTile;
    if (scan_tiles > c->sort.scan_tiles) {
      dev_alloc(c->sort.scan_lookback, scan_tiles);
      c->sort.scan_tiles = scan_tiles;
    }
    if (count > 0) {
      float* d_params = nullptr;
      float* d_sh = nullptr;
      dev_alloc(d_params, size_t(count) * 16);
      GS_CUDA_TRY(cudaMemcpyAsync(d_params, params16, sizeof(float) * 16 * count, cudaMemcpyHostToDevice, c->stream));
      if (sh_stride > 0) {
        dev_alloc(d_sh, size_t(count) * sh_stride);
        GS_CUDA_TRY(cudaMemcpyAsync(d_sh, sh, sizeof(float) * sh_stride * count, cudaMemcpyHostToDevice, c->stream));
      }
      gsk::launch_params_to_planes(d_params, d_sh, count, m, c->stream);
      GS_CUDA_TRY(cudaStreamSynchronize(c->stream));
      dev_free(d_params);
      dev_free(d_sh);
    }
    c->max_pairs_seen = 0;
    c->stepped = false;
    c->motion_nodes = 0;  // the binding was for the old slots
    c->motion_grad_ready = false;
    c->check_launch("gs_model_init");
    GS_CUDA_TRY(cudaStreamSynchronize(c->stream));
  });
}

int gs_model_info_get(gs_context* c, gs_model_info* out) {
  return guarded([&] {
    if (c == nullptr || out == nullptr) fail(GS_ERR_INVALID, "gs_model_info_get: null argument");
    out->capacity = c->model.cap;
    out->slots = c->model.slots;
    out->sh_stride = c->model.sh_stride;
    out->pair_capacity = c->pair_cap;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    out->device_bytes = total_b - free_b;
  });
}

int gs_model_export(gs_context* c, float* params16, float* sh, uint32_t max_slots, uint32_t* slots) {
  return guarded([&] {
    if (c == nullptr) fail(GS_ERR_INVALID, "gs_model_export: null context");
    if (slots) *slots = c->model.slots;
    const uint32_t n = std::min(max_slots, c->model.slots);
    if (n == 0) return;
    GS_CUDA_TRY(cudaSetDevice(c->device));
    if (params16)
      download_via<float>(c, size_t(n) * 16, params16, [&](float* tmp) {
        gsk::launch_planes_to_params(c->model, c->model.P, c->model.SH, tmp, nullptr, n, c->stream);
      });
    if (sh && c->model.sh_stride)
      download_via<float>(c, size_t(n) * c->model.sh_stride, sh, [&](float* tmp) {
        gsk::launch_planes_to_params(c->model, c->model.P, c->model.SH, nullptr, tmp, n, c->stream);
      });
  });
}

int gs_model_moments(gs_context* c, float* m16, float* v16, float* m_sh, float* v_sh) {
  return guarded([&] {
    if (c == nullptr) fail(GS_ERR_INVALID, "gs_model_moments: null context");
    const uint32_t n = c->model.slots;
    if (n == 0) return;
    GS_CUDA_TRY(cudaSetDevice(c->device));
    const gsk::Model& m = c->model;
    if (m16)
      download_via<float>(c, size_t(n) * 16, m16,
                          [&](float* t) { gsk::launch_planes_to_params(m, m.M, m.MSH, t, nullptr, n, c->stream); });
    if (v16)
      download_via<float>(c, size_t(n) * 16, v16,
                          [&](float* t) { gsk::launch_planes_to_params(m, m.V, m.VSH, t, nullptr, n, c->stream); });
    if (m_sh && m.sh_stride)
      download_via<float>(c, size_t(n) * m.sh_stride, m_sh,
                          [&](float* t) { gsk::launch_planes_to_params(m, m.M, m.MSH, nullptr, t, n, c->stream); });
    if (v_sh && m.sh_stride)
      download_via<float>(c, size_t(n) * m.sh_stride, v_sh,
                          [&](float* t) { gsk::launch_planes_to_params(m, m.V, m.VSH, nullptr, t, n, c->stream); });
  });
}

int gs_set_views(gs_context* c, uint32_t n_views, const gs_frame_data* frames, const uint8_t* const* rgba_targets) {
  return guarded([&] {
    if (c == nullptr || frames == nullptr) fail(GS_ERR_INVALID, "gs_set_views: null argument");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    c->set_views(n_views, frames, rgba_targets, nullptr);
  });
}

int gs_dataset_set(gs_context* c, uint32_t n_images, const uint32_t* widths, const uint32_t* heights,
                   const uint8_t* const* rgba) {
  return guarded([&] {
    if (c == nullptr || (n_images > 0 && (widths == nullptr || heights == nullptr || rgba == nullptr)))
      fail(GS_ERR_INVALID, "gs_dataset_set: null argument");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    c->set_dataset(n_images, widths, heights, rgba);
  });
}

int gs_set_views_dataset(gs_context* c, uint32_t n_views, const gs_frame_data* frames, const uint32_t* images) {
  return guarded([&] {
    if (c == nullptr || frames == nullptr || images == nullptr) fail(GS_ERR_INVALID, "gs_set_views_dataset: null argument");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    c->set_views(n_views, frames, nullptr, images);
  });
}

int gs_step(gs_context* c, uint32_t flags, gs_step_result* out) {
  return guarded([&] {
    if (c == nullptr) fail(GS_ERR_INVALID, "gs_step: null context");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    c->profile = (flags & GS_STEP_PROFILE) != 0u;
    c->count = (flags & GS_STEP_COUNT) != 0u;
    try {
      c->run_step((flags & GS_STEP_TRAIN) != 0u, out);
    } catch (...) {
      c->profile = c->count = false;
      throw;
    }
    c->profile = c->count = false;
  });
}

int gs_render(gs_context* c, const gs_frame_data* frame, uint8_t* rgba_out) {
  return guarded([&] {
    if (c == nullptr || frame == nullptr || rgba_out == nullptr) fail(GS_ERR_INVALID, "gs_render: null argument");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    gs_frame_data f = *frame;
    f.model[3] &= ~GS_FLAG_SSIM;
    c->set_views(1, &f, nullptr, nullptr);
    c->profile = false;
    c->run_step(false, nullptr, false);
    GS_CUDA_TRY(cudaMemcpy(rgba_out, c->image, size_t(f.image[0]) * f.image[1] * 4, cudaMemcpyDeviceToHost));
  });
}

int gs_densify(gs_context* c, const gs_frame_data* frame, uint32_t counters_out[4]) {
  return guarded([&] {
    if (c == nullptr || frame == nullptr) fail(GS_ERR_INVALID, "gs_densify: null argument");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    gs_frame_data f = *frame;
    f.model[0] = c->model.slots;
    f.model[2] = c->model.sh_stride;
    GS_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->h_table->frames[0] = f;
    GS_CUDA_TRY(cudaMemcpyAsync(c->d_table->frames, c->h_table->frames, sizeof(gs_frame_data), cudaMemcpyHostToDevice,
                                c->stream));
    int launches = 0;
    c->densify_slots = c->model.slots;
    gsk::launch_densify(c->d_table->frames, c->model, c->dens, c->sort, c->stream, &launches);
    uint32_t counters[4] = {0, 0, 0, 0};
    GS_CUDA_TRY(cudaStreamSynchronize(c->stream));
    GS_CUDA_TRY(cudaMemcpy(counters, c->dens.counters, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    c->check_launch("gs_densify");
    const uint32_t free_slots = counters[0], spawned = counters[1];
    const uint32_t room = free_slots + (c->model.cap - c->model.slots);
    const uint32_t placed = std::min(spawned, room);
    if (placed > free_slots) {
      c->model.slots += placed - free_slots;
      c->drop_graph();
    }
    counters[3] = c->model.slots;
    c->bind_motion();  // new gaussians need nodes (Trainer::after_step, trainer.cpp:944)
    if (counters_out) std::memcpy(counters_out, counters, sizeof(counters));
  });
}

int gs_reset_opacity(gs_context* c, float max_logit) {
  return guarded([&] {
    if (c == nullptr) fail(GS_ERR_INVALID, "gs_reset_opacity: null context");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    gsk::launch_reset_opacity(c->model, max_logit, c->stream);
    GS_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->check_launch("gs_reset_opacity");
  });
}

int gs_snapshot(gs_context* c, uint32_t view, gs_snapshot_kind which, void* host, size_t bytes, size_t* needed) {
  return guarded([&] {
    if (c == nullptr) fail(GS_ERR_INVALID, "gs_snapshot: null context");
    if (which != GS_SNAP_SPAWN && which != GS_SNAP_STATS && which != GS_SNAP_MOTION_BIND &&
        which != GS_SNAP_CONTRIBUTIONS &&
        (!c->stepped || view >= c->n_views))
      fail(GS_ERR_INVALID, "gs_snapshot: no such view in the latest step");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    GS_CUDA_TRY(cudaStreamSynchronize(c->stream));
    const gs_frame_data f = view < c->frames.size() ? c->frames[view] : gs_frame_data{};
    const size_t pixels = size_t(f.image[0]) * f.image[1];
    const size_t tiles = size_t(f.image[2]) * f.image[3];
    const uint32_t slots = c->model.slots, cap = c->model.cap;
    const uint64_t pairs = std::min<uint64_t>(c->last_pairs, c->pair_cap);
    const size_t pb = c->vt.pixel_base[view], tb = c->vt.tile_base[view];
    size_t size = 0;
    switch (which) {
      case GS_SNAP_PIXEL_COUNT: case GS_SNAP_IMAGE: case GS_SNAP_PIXEL_DOT: size = pixels * 4; break;
      case GS_SNAP_PIXEL_GRAD: case GS_SNAP_PIXEL_OUT: size = pixels * 16; break;
      case GS_SNAP_SPAWN: size = size_t(c->densify_slots) * 4; break;
      case GS_SNAP_PROJECTED: size = size_t(slots) * 64; break;
      case GS_SNAP_TILES: case GS_SNAP_OFFSETS: case GS_SNAP_DEPTH_KEY: size = size_t(slots) * 4; break;
      case GS_SNAP_STATS: size = size_t(slots) * 16; break;
      case GS_SNAP_CONTRIBUTIONS: size = sizeof(uint64_t); break;
      case GS_SNAP_MOTION_BIND:
        if (c->motion_nodes == 0u) fail(GS_ERR_INVALID, "gs_snapshot: no motion nodes");
        size = size_t(slots) * 32;
        break;
      case GS_SNAP_PAIR_GRADS: size = size_t(pairs) * 48; break;
      case GS_SNAP_PAIR_TILE: case GS_SNAP_RENDER_ORDER: case GS_SNAP_PAIR_GAUSSIAN: size = size_t(pairs) * 4; break;
      case GS_SNAP_RANGES: size = tiles * 8; break;
      case GS_SNAP_TILE_LOSS: size = tiles * 64; break;
      default: fail(GS_ERR_INVALID, "gs_snapshot: unknown buffer");
    }
    if (needed) *needed = size;
    if (host == nullptr) return;
    if (bytes < size) fail(GS_ERR_INVALID, "gs_snapshot: buffer too small");
    auto d2h = [&](void* dst, const void* src, size_t n) {
      if (n) GS_CUDA_TRY(cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost));
    };
    switch (which) {
      case GS_SNAP_PIXEL_COUNT: d2h(host, c->pixel_count + pb, size); break;
      case GS_SNAP_IMAGE: d2h(host, c->image + pb, size); break;
      case GS_SNAP_PIXEL_DOT: d2h(host, c->pixel_dot + pb, size); break;
      case GS_SNAP_PIXEL_GRAD: d2h(host, c->pixel_grad + pb, size); break;
      case GS_SNAP_PIXEL_OUT: d2h(host, c->pixel_out + pb, size); break;
      case GS_SNAP_SPAWN: d2h(host, c->dens.spawn, size); break;
      case GS_SNAP_TILES: d2h(host, c->vb.tiles + size_t(view) * cap, size); break;
      case GS_SNAP_OFFSETS:
        if (c->payload_gaussian)
          fail(GS_ERR_INVALID, "gs_snapshot: an atomic training step keeps no first-pair offsets: deterministic or "
                               "forward-only steps keep them");
        d2h(host, c->vb.offsets + size_t(view) * cap, size);
        break;
      case GS_SNAP_STATS: d2h(host, c->model.stats, size); break;
      case GS_SNAP_MOTION_BIND: d2h(host, c->motion_bind, size); break;
      case GS_SNAP_CONTRIBUTIONS: std::memcpy(host, &c->last_contributions, size); break;
      case GS_SNAP_TILE_LOSS: d2h(host, c->tile_loss + tb * 16, size); break;
      case GS_SNAP_PAIR_GRADS: d2h(host, c->pair_grads, size); break;
      case GS_SNAP_PAIR_GAUSSIAN: {
        if (c->payload_gaussian)
          fail(GS_ERR_INVALID, "gs_snapshot: an atomic training step sorts gaussians and keeps no per-pair gaussian: "
                               "deterministic or forward-only steps keep it");
        std::vector<uint32_t> g(pairs);
        d2h(g.data(), c->pair_gaussian, pairs * 4);
        for (auto& x : g) x -= view * cap;  // slots of this view
        std::memcpy(host, g.data(), size);
        break;
      }
      case GS_SNAP_PROJECTED:
        download_via<float>(c, size_t(slots) * 16, static_cast<float*>(host), [&](float* tmp) {
          gsk::launch_projected_record(c->vb, view, cap, slots, tmp, c->stream);
        });
        break;
      case GS_SNAP_RANGES: {
        std::vector<uint2> r(tiles);
        d2h(r.data(), c->ranges + tb, tiles * 8);
        // View-local positions: the view's pairs start at its first non-empty tile.
        uint32_t first = UINT32_MAX;
        for (const uint2& x : r)
          if (x.y > x.x) first = std::min(first, x.x);
        for (uint2& x : r) {
          if (x.y > x.x) {
            x.x -= first;
            x.y -= first;
          } else {
            x = make_uint2(0u, 0u);
          }
        }
        std::memcpy(host, r.data(), size);
        break;
      }
      case GS_SNAP_PAIR_TILE: case GS_SNAP_RENDER_ORDER: {
        if (c->payload_gaussian)
          fail(GS_ERR_INVALID, "gs_snapshot: an atomic training step sorts gaussians, not pair indices: the pair "
                               "tiles and the render order are kept by deterministic or forward-only steps");
        std::vector<uint32_t> k(pairs), v(pairs);
        d2h(k.data(), c->sorted_keys, pairs * 4);
        d2h(v.data(), c->sorted_values, pairs * 4);
        uint32_t* o = static_cast<uint32_t*>(host);
        if (which == GS_SNAP_RENDER_ORDER) {
          std::memcpy(o, v.data(), size);
        } else {
          for (uint64_t p = 0; p < pairs; ++p) o[p] = ~0u;
          for (uint64_t s = 0; s < pairs; ++s)
            if (v[s] < pairs) o[v[s]] = k[s] - uint32_t(tb);
        }
        break;
      }
      case GS_SNAP_DEPTH_KEY: {
        const size_t n = size_t(c->n_views) * slots;
        std::vector<uint32_t> k(n), v(n);
        d2h(k.data(), c->depth_sorted_keys, n * 4);
        d2h(v.data(), c->depth_sorted_vals, n * 4);
        uint32_t* o = static_cast<uint32_t*>(host);
        for (uint32_t i = 0; i < slots; ++i) o[i] = ~0u;
        for (size_t e = 0; e < n; ++e)
          if (v[e] / cap == view && v[e] % cap < slots) o[v[e] % cap] = k[e] & 0xffffu;
        break;
      }
      default: break;
    }
  });
}

int gs_motion_nodes(gs_context* c, uint32_t count, const float* nodes4) {
  return guarded([&] {
    if (c == nullptr) fail(GS_ERR_INVALID, "gs_motion_nodes: null context");
    if (count > GS_MAX_MOTION_NODES) fail(GS_ERR_INVALID, "gs_motion_nodes: at most 128 nodes");
    if (count > 0 && nodes4 == nullptr) fail(GS_ERR_INVALID, "gs_motion_nodes: null nodes");
    if (c->model.cap == 0) fail(GS_ERR_INVALID, "gs_motion_nodes: no model (gs_model_init first)");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    GS_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->drop_graph();
    c->motion_grad_ready = false;
    c->motion_nodes = 0;
    if (count == 0) return;
    if (c->motion_rest == nullptr) {
      dev_alloc(c->motion_rest, gsk::kMaxMotionNodes);
      dev_alloc(c->d_motion_views, size_t(GS_MAX_VIEWS) * gsk::kMaxMotionNodes);
      dev_alloc(c->d_motion_grad, size_t(GS_MAX_VIEWS) * gsk::kMaxMotionNodes * 8);
      const size_t table = sizeof(gsk::MotionNode) * GS_MAX_VIEWS * gsk::kMaxMotionNodes;
      GS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&c->h_motion_views), table));
      std::memset(c->h_motion_views, 0, table);
      const size_t grads = sizeof(double) * GS_MAX_VIEWS * gsk::kMaxMotionNodes * 8;
      GS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&c->h_motion_grad), grads));
      std::memset(c->h_motion_grad, 0, grads);
    }
    if (c->motion_bind_cap < c->model.cap) {
      dev_alloc(c->motion_bind, size_t(c->model.cap) * 2);
      c->motion_bind_cap = c->model.cap;
    }
    GS_CUDA_TRY(cudaMemcpy(c->motion_rest, nodes4, sizeof(float4) * count, cudaMemcpyHostToDevice));
    c->motion_nodes = count;
    c->bind_motion();
  });
}

int gs_motion_bind(gs_context* c) {
  return guarded([&] {
    if (c == nullptr) fail(GS_ERR_INVALID, "gs_motion_bind: null context");
    if (c->motion_nodes == 0u) fail(GS_ERR_INVALID, "gs_motion_bind: no motion nodes (gs_motion_nodes first)");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    GS_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->bind_motion();
  });
}

int gs_set_view_motion(gs_context* c, uint32_t view, const float* nodes20) {
  return guarded([&] {
    if (c == nullptr || nodes20 == nullptr) fail(GS_ERR_INVALID, "gs_set_view_motion: null argument");
    if (view >= GS_MAX_VIEWS) fail(GS_ERR_INVALID, "gs_set_view_motion: view out of range");
    if (c->motion_nodes == 0u) fail(GS_ERR_INVALID, "gs_set_view_motion: no motion nodes (gs_motion_nodes first)");
    std::memcpy(c->h_motion_views + size_t(view) * gsk::kMaxMotionNodes, nodes20,
                sizeof(gsk::MotionNode) * c->motion_nodes);
  });
}

int gs_motion_gradient(gs_context* c, uint32_t view, double* out, uint32_t count) {
  return guarded([&] {
    if (c == nullptr || out == nullptr) fail(GS_ERR_INVALID, "gs_motion_gradient: null argument");
    if (!c->motion_grad_ready || view >= c->n_views)
      fail(GS_ERR_INVALID, "gs_motion_gradient: the latest step computed no motion gradient for this view");
    if (count > c->motion_nodes) fail(GS_ERR_INVALID, "gs_motion_gradient: more nodes than there are");
    for (uint32_t k = 0; k < count; ++k)
      for (int j = 0; j < 6; ++j) out[k * 6 + j] = c->h_motion_grad[(size_t(view) * gsk::kMaxMotionNodes + k) * 8 + j];
  });
}

int gs_set_tuning(gs_context* c, const gs_tuning* t) {
  return guarded([&] {
    if (c == nullptr || t == nullptr) fail(GS_ERR_INVALID, "gs_set_tuning: null argument");
    if (t->forward_pixels != 0 && t->forward_pixels != 1 && t->forward_pixels != 2 && t->forward_pixels != 4)
      fail(GS_ERR_INVALID, "gs_set_tuning: forward_pixels must be 1, 2 or 4");
    if (t->backward_pixels != 0 && t->backward_pixels != 1 && t->backward_pixels != 2 && t->backward_pixels != 4 &&
        t->backward_pixels != 8)
      fail(GS_ERR_INVALID, "gs_set_tuning: backward_pixels must be 1, 2, 4 or 8");
    if (t->backward_batch != 0 && t->backward_batch != 32 && t->backward_batch != 64)
      fail(GS_ERR_INVALID, "gs_set_tuning: backward_batch must be 32 or 64");
    if (t->sort_digit_bits != 0 && (t->sort_digit_bits < 4 || t->sort_digit_bits > 8))
      fail(GS_ERR_INVALID, "gs_set_tuning: sort_digit_bits must be 4..8");
    if (t->forward_batch != 0 && t->forward_batch != 64 && t->forward_batch != 128 && t->forward_batch != 256)
      fail(GS_ERR_INVALID, "gs_set_tuning: forward_batch must be 64, 128 or 256");
    c->tuning = *t;
    if (c->tuning.min_pair_capacity == 0) c->tuning.min_pair_capacity = 1;
    c->drop_graph();
  });
}

int gs_get_tuning(gs_context* c, gs_tuning* t) {
  return guarded([&] {
    if (c == nullptr || t == nullptr) fail(GS_ERR_INVALID, "gs_get_tuning: null argument");
    *t = c->tuning;
  });
}

int gs_autotune(gs_context* c, uint32_t steps_per_candidate, gs_tuning* chosen) {
  return guarded([&] {
    if (c == nullptr) fail(GS_ERR_INVALID, "gs_autotune: null context");
    GS_CUDA_TRY(cudaSetDevice(c->device));
    c->profile = false;
    c->autotune(std::max(1u, steps_per_candidate));
    if (chosen != nullptr) *chosen = c->tuning;
  });
}

}  // extern "C"
