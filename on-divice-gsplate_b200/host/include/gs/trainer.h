// The training loop on the B200 path: the reference engine's gs::Trainer
// (engine/include/gs/trainer.h:20-330) over libgs_cuda's C ABI.
//
// The public API keeps the reference's names, argument meanings and error behaviour
// (std::runtime_error from the constructor when the device cannot train; overflowing pair
// buffers are grown and the step re-run, not an error). The GPU work of a step, the
// buffers and their growth live in libgs_cuda; this class keeps the host side: view order,
// backgrounds, learning-rate, SH-degree and loss-weight schedules, densification and
// opacity-reset schedules, statistics, evaluation and export.
//
// Camera pose refinement, exposure refinement, subject motion and head weighting follow
// the reference (trainer.cpp:1164-1771; trainer.h:60-131): pose corrections per training
// view by Adam on the pose gradient the step sums on the GPU, held-out views aligned
// before evaluation, per-view colour gains fitted from the forward pass's sums, per-view
// rigid motions of control nodes the gaussians follow (SC-GS), and the head region's
// pixels weighted in the loss.
//
// Extensions: `views_per_step` > 1 renders and differentiates that many views in one
// launch per pass and takes one Adam step on their summed gradients (batched training;
// a step still counts one iteration; each view still gets its own pose gradient and gain
// fit), and the retune steps run gs_autotune, which picks pixels per thread, the backward
// batch and the sort digit width.
#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <random>
#include <string>
#include <utility>
#include <vector>

#include "gs/camera.h"
#include "gs/dataset.h"
#include "gs/splat_scene.h"

struct gs_context;
struct gs_frame_data;
struct gs_step_result;

namespace gs {

// The role of the reference's VkContext& (device + stream owner): which CUDA device the
// trainer's libgs_cuda context is created on.
struct CudaContext {
  int device = 0;
};

struct TrainOptions {
  uint32_t iterations = 3000;
  uint32_t max_gaussians = 300000;  // slot capacity
  int sh_degree = 3;
  uint32_t sh_degree_interval = 500;  // the active SH degree goes up by one every this many steps
  bool masked = true;                 // composite masked targets over the background (datasets with masks)
  bool random_background = true;      // otherwise `background`
  float background[3] = {0.0f, 0.0f, 0.0f};
  float lr_position = 1.6e-4f;  // times the camera extent, decaying exponentially to lr_position_final
  float lr_position_final = 1.6e-6f;
  float lr_scale = 5e-3f;
  float lr_rotation = 1e-3f;
  float lr_opacity = 2.5e-2f;
  float lr_sh_dc = 2.5e-3f;
  float lr_sh_rest = 2.5e-3f / 20.0f;
  float lambda_dssim = 0.2f;     // loss (1 - lambda) L1 + lambda (1 - SSIM), lambda ramping
  float lambda_dssim_end = 1.0f;  // to this by the last step (< 0: no ramp)
  // Pixels in the head region (estimate_head) weigh this much in the loss; views where the
  // head covers much of the frame (radius >= a quarter of the height) are left at 1.
  HeadRegion head;
  float head_weight = 1.0f;
  // Camera pose refinement (trainer.h:69-81): from step pose_from each training view's
  // pose correction takes an Adam step on its pose gradient; held-out views are aligned
  // with eval_pose_steps steps that move only their camera before evaluation.
  bool refine_poses = false;
  uint32_t pose_from = 300;
  float lr_pose_shift = 1e-3f;    // per update, times the camera extent
  float lr_pose_turn = 1e-3f;     // radians per update
  float lr_pose_final = 1.0f;     // the rates decay exponentially to this fraction by the last step
  uint32_t eval_pose_steps = 8;
  float eval_pose_step = 0.005f;  // the alignment's first step, times the camera extent
  // Subject motion (trainer.h:83-117): `motion_nodes` control nodes spread over the
  // initial gaussians (k-means); in each training view every node moves rigidly (a turn
  // about itself and a shift) and each gaussian follows its 4 nearest nodes. The motions
  // are trained by Adam from step motion_from, kept small (motion_decay), alike between
  // neighbouring nodes (motion_rigidity) and neighbouring views (motion_smoothness), and
  // centred on the rest pose over the views (motion_center); penalties in units of the
  // node spacing. The model stays the subject at rest; held-out views take the motion of
  // the training views next to them.
  bool refine_motion = false;
  uint32_t motion_nodes = 64;     // at most 128
  uint32_t motion_from = 300;
  float lr_motion_shift = 2e-3f;  // per update, times the camera extent
  float lr_motion_turn = 3e-3f;   // radians per update
  float lr_motion_final = 0.1f;   // the rates decay exponentially to this fraction by the last step
  float motion_decay = 1e-4f;
  float motion_rigidity = 1e-3f;
  float motion_smoothness = 1e-2f;
  float motion_center = 1e-2f;
  // Exposure refinement (trainer.h:121-131): per-view colour gains fitted from the
  // forward pass's sums, blended in at exposure_rate from step exposure_from, used
  // divided by their geometric mean over the trained views.
  bool refine_exposure = false;
  uint32_t exposure_from = 300;
  float exposure_rate = 0.3f;
  bool sparse_adam = false;       // gaussians that drew nothing in a step keep their values and moments
  uint32_t densify_from = 300;
  uint32_t densify_until = 2000;
  uint32_t densify_interval = 100;
  uint32_t opacity_reset_interval = 0;  // 0 disables
  float densify_grad_threshold = 2e-4f;
  float percent_dense = 0.01f;  // clone below, split above this fraction of the extent
  float prune_opacity = 0.005f;
  // Retuning: at step retune_first and every retune_interval steps (0: never) gs_autotune
  // times the candidate tunings on training steps and keeps the fastest.
  uint32_t retune_first = 20;
  uint32_t retune_interval = 500;
  bool autotune = true;
  bool deterministic = true;  // fixed-order gradient sums (bit-stable); false: atomics
  uint32_t views_per_step = 1;  // batched training: views rendered and differentiated per Adam step (1..16)
  uint32_t min_pair_capacity = 1 << 16;
  uint64_t initial_pair_guess = 0;  // pairs to allocate for before the first count (0: four per gaussian)
  uint32_t seed = 1;
};

// The defaults' schedule (densification, opacity reset, SH degree) scaled to `iterations`
// (trainer.cpp:133-145).
TrainOptions scaled_options(uint32_t iterations);

// GPU milliseconds of each pass in one profiled step.
struct PassTimes {
  double project = 0.0;    // projection + pair count
  double sort = 0.0;       // depth sort, scan, pair emission, pair sort, tile ranges
  double rasterize = 0.0;  // forward + L1 loss
  double ssim = 0.0;       // SSIM and its gradient
  double backward = 0.0;   // per-pair gradients
  double optimize = 0.0;   // pair sums, projection backward, Adam
  bool valid = false;
};

struct TrainStats {
  uint32_t step = 0;
  uint32_t gaussians = 0;  // alive
  uint32_t slots = 0;      // slots in use (alive + free)
  uint64_t pairs = 0;      // (tile, gaussian) pairs of the last step (all its views)
  double l1 = 0.0;         // mean absolute error of the last step's views
  double psnr = 0.0;       // of the last step's views (their mean)
  double ssim = 0.0;       // of the last step's views (0 when not computed)
  double loss = 0.0;       // the training loss of the last step's views
  double step_ms = 0.0;    // exponential moving average of the wall-clock step time
  int sh_degree = 0;       // active
  uint32_t densify_events = 0;
  uint32_t spawned = 0;
  uint32_t pruned = 0;
  uint32_t tile_mismatch = 0;   // gaussians whose emitted tiles differed from the count (0)
  uint32_t overflow_steps = 0;  // steps whose pairs did not fit (their update was skipped)
  uint64_t views = 0;           // training views processed
  double pose_shift_mean = 0.0, pose_shift_max = 0.0;  // dataset units
  double pose_turn_mean = 0.0, pose_turn_max = 0.0;    // degrees
  uint32_t pose_updates = 0;
  double exposure_low = 1.0, exposure_high = 1.0, exposure_tint = 0.0;  // 5th/95th percentile luminance gain
  uint32_t exposure_updates = 0;
  uint32_t motion_nodes = 0;
  double motion_shift_mean = 0.0, motion_shift_max = 0.0;  // dataset units
  double motion_turn_mean = 0.0, motion_turn_max = 0.0;    // degrees
  uint32_t motion_updates = 0;                             // view updates
  struct Timing {
    double wall_ms = 0.0;  // moving averages per step
    double gpu_ms = 0.0;
    double batch = 0.0;    // views per step
  } timing;
};

struct RetuneResult {
  uint32_t step = 0;
  std::string chosen;  // "fpx=2 fbatch=256 bpx=4 batch=64 digits=8 sync deterministic"
};

struct EvalResult {
  double psnr = 0.0;  // mean over the held-out views (aligned first when refining poses)
  bool aligned = false;
  double psnr_unaligned = 0.0;  // at the poses as given, when aligned
  double ssim = 0.0;
  double head_psnr = 0.0;
  uint32_t head_views = 0;
  double l1 = 0.0;
  uint32_t views = 0;
};

class Trainer {
 public:
  // Throws std::runtime_error if the device cannot train (or a feature this path does not
  // have is asked for). Takes the dataset by value: move it in to avoid a copy.
  Trainer(CudaContext& ctx, Dataset dataset, const SplatScene& initial, const TrainOptions& options);
  ~Trainer();
  Trainer(const Trainer&) = delete;
  Trainer& operator=(const Trainer&) = delete;

  // One optimisation step on the next training view(s), then densification on schedule.
  // With `profile`, the passes are timed (last_profile()).
  void step(bool profile = false);
  // Up to `count` steps (fewer at the end); returns the steps run.
  uint32_t steps(uint32_t count);
  const PassTimes& last_profile() const { return profile_; }
  bool finished() const { return stats_.step >= options_.iterations; }
  const TrainStats& stats() const { return stats_; }
  const TrainOptions& options() const { return options_; }
  const Dataset& dataset() const { return dataset_; }

  // The current model (at rest) from `camera` over `background`: RGBA8, alpha = coverage.
  std::vector<uint8_t> render(const Camera& camera, const float background[3]);
  // Held-out views over a black background (with the subject's motion interpolated from
  // the views next to them, when refining motion).
  EvalResult evaluate();
  // View `frame` as its camera saw it: with its pose correction and, when refining
  // motion, the subject's motion then.
  std::vector<uint8_t> render_view(size_t frame, const float background[3]);
  // The held-out views of another dataset of the same subject standing still (a twin
  // capture): the model at rest against it, gains 1, no motion (trainer.h:283).
  EvalResult evaluate_at_rest(const Dataset& other);
  // A view's camera with its pose correction (the dataset's pose without refinement).
  Camera camera_for(size_t frame) const;
  // A view's exposure gains (the photo is divided by them): centred, interpolated for views
  // not trained on, 1 without refine_exposure.
  void view_gain(size_t frame, float gain[3]) const;
  // The alive gaussians, in the dataset's world.
  SplatScene export_scene();

  // Testing: one step on `frame` over `background`. With all learning rates zero the
  // parameters stay put and first_step_gradients() returns the first step's gradients.
  void step_on(size_t frame, const float background[3], bool profile = false);
  struct Gradients {
    std::vector<float> params;  // 16 per slot
    std::vector<float> sh;      // sh_stride() per slot
  };
  Gradients first_step_gradients();
  // The pose gradient of the latest pose update: dL/dd xyz, dL/dw xyz.
  const double* last_pose_gradient() const { return last_pose_grad_; }

  // Subject motion: the control nodes at rest (empty without refine_motion).
  struct MotionNode {
    float position[3];
    float radius;  // gaussians weigh it by exp(-d^2 / (2 radius^2))
  };
  const std::vector<MotionNode>& motion_nodes() const { return nodes_; }
  // A node's motion in view `frame`: turn (axis-angle, radians) and shift.
  void node_motion(size_t frame, uint32_t node, float turn[3], float shift[3]) const;
  // Testing: sets it (the view then counts as trained).
  void set_node_motion(size_t frame, uint32_t node, const float turn[3], const float shift[3]);
  // Testing: the motion gradient of the latest motion update (image loss only), 6 per
  // node: dL/dshift xyz, dL/dturn xyz (world axes).
  const std::vector<double>& last_motion_gradient() const { return last_motion_grad_; }
  // Testing: each slot's 4 nodes and weights.
  struct MotionBinding {
    std::vector<uint32_t> nodes;
    std::vector<float> weights;
  };
  MotionBinding motion_binding();
  struct DebugSnapshot {
    std::vector<uint32_t> pixel_count;
    std::vector<float> pixel_grad;
    std::vector<float> projected;
    std::vector<uint32_t> tiles;
    std::vector<uint32_t> offsets;
    std::vector<float> pair_grads;
    std::vector<uint32_t> pair_tile;
    std::vector<uint32_t> render_order;
    std::vector<uint32_t> depth_key;
  };
  DebugSnapshot debug_snapshot();
  uint32_t sh_stride() const { return sh_stride_; }
  // The tuning in use ("fpx=2 fbatch=256 bpx=4 batch=64 digits=8 sync deterministic"), in place of the
  // reference's backward-variant name.
  std::string reduction() const;
  // Testing: runs the backward (and the passes it shares knobs with) under the tuning
  // `name` names, in reduction()'s form: any of fpx=1|2|4, fbatch=64|128|256, bpx=1|2|4,
  // batch=32|64, digits=4..8, sync|async and deterministic|atomic, the others kept (trainer.h:324 picks a backward
  // variant by name). False, and nothing changed, for a name it cannot parse.
  bool select_backward(const std::string& name);
  const std::vector<RetuneResult>& retunes() const { return retunes_; }

 private:
  // Pose, exposure and subject-motion state: the capture order, the camera corrections,
  // the gains and the node rig (host/src/refinement.h, host/src/node_rig.h).
  struct Corrections;

  void next_view(size_t& frame, float background[3]);
  void run_step(const std::vector<size_t>& frames, const std::vector<std::array<float, 3>>& backgrounds,
                bool profile);
  void write_frame(gs_frame_data& f, const Camera& camera, const float background[3], uint32_t step, bool ssim,
                   bool masked, uint32_t flags = 0u, const float* gain = nullptr) const;
  // One held-out measurement (forward only) or alignment probe of `camera` against the
  // dataset's image `frame` (or `rgba`, another dataset's, when not null) over black; with
  // `moved` (a node table, gs_set_view_motion's layout) the subject moves by it.
  void run_eval_view(const Camera& camera, size_t frame, const uint8_t* rgba, const float gain[3], uint32_t flags,
                     const std::vector<float>* moved, gs_step_result& r);
  EvalResult evaluate_views(const Dataset& ds, bool own);
  std::vector<uint8_t> render_with(const Camera& camera, const float background[3], const std::vector<float>* moved);
  // Subject motion (trainer_refine.cpp).
  void build_rig(const SplatScene& initial);  // the nodes over the initial gaussians, then gs_motion_nodes
  void bind_motion();                         // gs_motion_bind
  bool refines_motion_at(uint32_t step) const;
  bool moves_subject() const;                 // some view's motion has been learned
  std::vector<float> motion_table(size_t frame) const;  // its node table (estimated when not learned)
  void upload_motion(uint32_t view, const std::vector<float>& table);
  // Pose and exposure (trainer_refine.cpp).
  bool refines_pose_at(uint32_t step) const { return options_.refine_poses && step >= options_.pose_from; }
  bool refines_exposure_at(uint32_t step) const {
    return options_.refine_exposure && step >= options_.exposure_from;
  }
  double rate_fade(float final_fraction) const;  // final_fraction ^ (step / iterations)
  // After a training step that kept its update: each view's pose, gain and motion learn
  // from the step's gradients and sums; the spreads in the statistics follow.
  void learn_corrections(const std::vector<size_t>& frames, const gs_step_result& r, bool pose, bool exposure,
                         bool motion);
  // A held-out view's camera aligned to its image (evaluate_views): the correction found,
  // applied to `given`.
  Camera align_view(const Camera& given, size_t frame, const uint8_t* rgba, const float gain[3],
                    const std::vector<float>* moved, bool own);
  uint32_t sh_degree_at(uint32_t step) const;
  double lambda_at(uint32_t step) const;
  bool uses_ssim() const;
  void after_step();
  void densify();
  void reset_opacity();
  bool retune_due(uint32_t s) const;
  void check(int code, const char* what) const;

  CudaContext& ctx_;
  gs_context* gpu_ = nullptr;
  Dataset dataset_;
  TrainOptions options_;
  uint32_t sh_stride_ = 0;
  uint32_t capacity_ = 0;
  std::vector<size_t> train_frames_, order_;
  size_t order_pos_ = 0;
  std::mt19937 rng_;
  TrainStats stats_;
  PassTimes profile_;
  std::vector<RetuneResult> retunes_;
  std::vector<uint8_t> frame_bytes_;  // the last step's first FrameData (densify thresholds)
  std::unique_ptr<Corrections> fix_;
  std::vector<MotionNode> nodes_;          // the rig's nodes, as motion_nodes() reports them
  double last_pose_grad_[6] = {0, 0, 0, 0, 0, 0};
  std::vector<double> last_motion_grad_;
  uint32_t bound_at_ = 0;  // step of the latest binding
};

}  // namespace gs
