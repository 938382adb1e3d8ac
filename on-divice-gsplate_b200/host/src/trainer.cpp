// gs::Trainer over libgs_cuda. The host side of engine/src/trainer.cpp: view order
// (next_view, :911-924), FrameData (write_frame, :440-547), statistics (read_slot /
// set_view_stats, :778-805), the densify and opacity-reset schedule (after_step,
// :932-945; densify, :1083-1119; reset_opacity, :1121-1128), evaluation (evaluate_views,
// :1244-1292) and export (export_scene, :1773-1800). Pose and exposure refinement and
// subject motion are in trainer_refine.cpp.
#include "gs/trainer.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "corrections.h"
#include "frame.h"
#include "gs_cuda.h"

namespace gs {

namespace {

constexpr float kBeta1 = 0.9f;  // trainer.cpp:68

struct ViewLosses {
  double l1 = 0, psnr = 0, ssim = 0, loss = 0;
};

// One view's statistics from its loss sums (set_view_stats, trainer.cpp:797-805).
ViewLosses view_losses(const double* s, uint32_t width, uint32_t height, double lambda, bool ssim) {
  const double n = 3.0 * width * height;
  ViewLosses v;
  v.l1 = s[0] / n;
  v.psnr = -10.0 * std::log10(std::max(s[1] / n, 1e-12));
  v.ssim = ssim ? s[2] / n : 0.0;
  v.loss = ((1.0 - lambda) * s[3] + lambda * (s[5] - s[4])) / n;
  return v;
}

}  // namespace

TrainOptions scaled_options(uint32_t iterations) {
  TrainOptions o;
  const double scale = double(iterations) / double(o.iterations);
  o.iterations = iterations;
  o.densify_from = uint32_t(o.densify_from * scale);
  o.densify_until = uint32_t(o.densify_until * scale);
  o.opacity_reset_interval = uint32_t(o.opacity_reset_interval * scale);
  o.sh_degree_interval = std::max(1u, uint32_t(o.sh_degree_interval * scale));
  return o;
}

void Trainer::check(int code, const char* what) const { detail::check_status(code, what); }

Trainer::Trainer(CudaContext& ctx, Dataset dataset, const SplatScene& initial, const TrainOptions& options)
    : ctx_(ctx), dataset_(std::move(dataset)), options_(options), rng_(options.seed) {
  if (dataset_.frames.empty() || dataset_.width == 0) throw std::runtime_error("Trainer: empty dataset");
  if (options_.views_per_step < 1 || options_.views_per_step > GS_MAX_VIEWS)
    throw std::runtime_error("Trainer: views_per_step must be 1.." + std::to_string(GS_MAX_VIEWS));
  if (options_.sh_degree < 0 || options_.sh_degree > 3) throw std::runtime_error("Trainer: sh_degree must be 0..3");
  for (size_t i = 0; i < dataset_.frames.size(); ++i) {
    const DatasetFrame& f = dataset_.frames[i];
    const Camera c = dataset_camera(dataset_, f);
    if (f.rgba.size() != size_t(c.width) * c.height * 4)
      throw std::runtime_error("Trainer: frame " + f.name + " has the wrong image size");
    if (!f.holdout) train_frames_.push_back(i);
  }
  if (train_frames_.empty()) throw std::runtime_error("Trainer: no training frames");
  fix_ = std::make_unique<Corrections>();
  fix_->order.build(dataset_.frames.size(), train_frames_);
  fix_->poses.reset(dataset_.frames.size());
  fix_->gains.reset(dataset_.frames.size());
  sh_stride_ = uint32_t(sh_rest_coeffs(options_.sh_degree) * 3);
  capacity_ = std::max(std::max(options_.max_gaussians, initial.count), 1u);

  check(gs_create(ctx_.device, &gpu_), "Trainer: gs_create");
  try {
    std::vector<float> p, s;
    detail::pack_params(initial, options_.sh_degree, sh_stride_, p, s);
    check(gs_model_init(gpu_, capacity_, sh_stride_, p.data(), sh_stride_ ? s.data() : nullptr, initial.count),
          "Trainer: gs_model_init");
    gs_tuning t;
    check(gs_get_tuning(gpu_, &t), "Trainer: gs_get_tuning");
    t.deterministic = options_.deterministic ? 1u : 0u;
    t.min_pair_capacity = options_.min_pair_capacity;
    t.initial_pairs = options_.initial_pair_guess;
    t.retry = 1u;
    t.graph = 1u;
    check(gs_set_tuning(gpu_, &t), "Trainer: gs_set_tuning");
    // The dataset's images stay in HBM for the whole run.
    std::vector<uint32_t> w, h;
    std::vector<const uint8_t*> ptr;
    for (const DatasetFrame& f : dataset_.frames) {
      const Camera c = dataset_camera(dataset_, f);
      w.push_back(c.width);
      h.push_back(c.height);
      ptr.push_back(f.rgba.data());
    }
    check(gs_dataset_set(gpu_, uint32_t(ptr.size()), w.data(), h.data(), ptr.data()), "Trainer: gs_dataset_set");
    if (options_.refine_motion) build_rig(initial);
  } catch (...) {
    gs_destroy(gpu_);
    gpu_ = nullptr;
    throw;
  }
  stats_.slots = initial.count;
  stats_.gaussians = initial.count;
}

Trainer::~Trainer() {
  if (gpu_ != nullptr) gs_destroy(gpu_);
}

uint32_t Trainer::sh_degree_at(uint32_t step) const {
  return std::min<uint32_t>(uint32_t(options_.sh_degree),
                            options_.sh_degree_interval > 0 ? step / options_.sh_degree_interval
                                                            : uint32_t(options_.sh_degree));
}

double Trainer::lambda_at(uint32_t step) const {
  if (options_.lambda_dssim_end < 0.0f || options_.iterations <= 1) return options_.lambda_dssim;
  const float t = std::min(1.0f, float(step) / float(options_.iterations - 1));
  return options_.lambda_dssim + (options_.lambda_dssim_end - options_.lambda_dssim) * t;
}

bool Trainer::uses_ssim() const { return options_.lambda_dssim > 0.0f || options_.lambda_dssim_end > 0.0f; }

void Trainer::write_frame(gs_frame_data& f, const Camera& camera, const float background[3], uint32_t step,
                          bool ssim, bool masked, uint32_t flags, const float* gain) const {
  flags |= (masked ? GS_FLAG_MASKED_TARGET : 0u) | (ssim ? GS_FLAG_SSIM : 0u) |
           (options_.sparse_adam ? GS_FLAG_SPARSE_ADAM : 0u);
  detail::frame_geometry(f, camera, stats_.slots, sh_stride_, int(sh_degree_at(step)), flags, background);
  detail::frame_schedule(f, options_, step, dataset_.camera_extent, float(lambda_at(step)));
  detail::frame_refinement(f, camera, options_.head, options_.head_weight, gain);
}

void Trainer::next_view(size_t& frame, float background[3]) {
  if (order_pos_ >= order_.size()) {
    order_ = train_frames_;
    std::shuffle(order_.begin(), order_.end(), rng_);
    order_pos_ = 0;
  }
  if (options_.random_background) {
    std::uniform_real_distribution<float> u(0.0f, 1.0f);
    for (int c = 0; c < 3; ++c) background[c] = u(rng_);
  } else {
    std::copy(options_.background, options_.background + 3, background);
  }
  frame = order_[order_pos_++];
}

bool Trainer::retune_due(uint32_t s) const {
  return options_.autotune && s < options_.iterations &&
         (s == options_.retune_first || (options_.retune_interval > 0 && s > 0 && s % options_.retune_interval == 0));
}

std::string Trainer::reduction() const {
  gs_tuning t;
  if (gs_get_tuning(gpu_, &t) != GS_OK) return "unknown";
  return "fpx=" + std::to_string(t.forward_pixels) + " fbatch=" + std::to_string(t.forward_batch) +
         " bpx=" + std::to_string(t.backward_pixels) + " batch=" + std::to_string(t.backward_batch) +
         " digits=" + std::to_string(t.sort_digit_bits) + (t.stage_async ? " async" : " sync") +
         (t.deterministic ? " deterministic" : " atomic");
}

bool Trainer::select_backward(const std::string& name) {
  gs_tuning t;
  if (gs_get_tuning(gpu_, &t) != GS_OK) return false;
  size_t pos = 0;
  while (pos < name.size()) {
    const size_t end = std::min(name.find(' ', pos), name.size());
    const std::string word = name.substr(pos, end - pos);
    pos = end + 1;
    if (word.empty()) continue;
    if (word == "deterministic" || word == "atomic") {
      t.deterministic = word == "deterministic" ? 1u : 0u;
      continue;
    }
    if (word == "async" || word == "sync") {
      t.stage_async = word == "async" ? 1u : 0u;
      continue;
    }
    const size_t eq = word.find('=');
    if (eq == std::string::npos) return false;
    const std::string key = word.substr(0, eq);
    char* rest = nullptr;
    const unsigned long v = std::strtoul(word.c_str() + eq + 1, &rest, 10);
    if (rest == word.c_str() + eq + 1 || *rest != '\0') return false;
    if (key == "fpx" && (v == 1 || v == 2 || v == 4)) t.forward_pixels = uint32_t(v);
    else if (key == "fbatch" && (v == 64 || v == 128 || v == 256)) t.forward_batch = uint32_t(v);
    else if (key == "bpx" && (v == 1 || v == 2 || v == 4 || v == 8)) t.backward_pixels = uint32_t(v);
    else if (key == "batch" && (v == 32 || v == 64)) t.backward_batch = uint32_t(v);
    else if (key == "digits" && v >= 4 && v <= 8) t.sort_digit_bits = uint32_t(v);
    else return false;
  }
  return gs_set_tuning(gpu_, &t) == GS_OK;
}

void Trainer::run_step(const std::vector<size_t>& frames, const std::vector<std::array<float, 3>>& backgrounds,
                       bool profile) {
  const auto start = std::chrono::steady_clock::now();
  const uint32_t step = stats_.step;
  const bool ssim = uses_ssim();
  const uint32_t k = uint32_t(frames.size());
  std::vector<gs_frame_data> fd(k);
  std::vector<uint32_t> images(k);
  std::vector<Camera> cams(k);
  const bool pose = refines_pose_at(step), exposure = refines_exposure_at(step), motion = refines_motion_at(step);
  for (uint32_t v = 0; v < k; ++v) {
    cams[v] = camera_for(frames[v]);
    float gain[3];
    view_gain(frames[v], gain);
    if (motion) fix_->rig.begin(frames[v], fix_->order);
    const uint32_t flags =
        (pose ? GS_FLAG_POSE_GRAD : 0u) | (motion ? GS_FLAG_MOTION | GS_FLAG_MOTION_GRAD : 0u);
    write_frame(fd[v], cams[v], backgrounds[v].data(), step, ssim, options_.masked, flags, gain);
    images[v] = uint32_t(frames[v]);
  }
  check(gs_set_views_dataset(gpu_, k, fd.data(), images.data()), "Trainer::step: gs_set_views_dataset");
  if (motion)
    for (uint32_t v = 0; v < k; ++v) upload_motion(v, fix_->rig.table(fix_->rig.pose(frames[v])));
  if (retune_due(step)) {
    gs_tuning chosen;
    check(gs_autotune(gpu_, 2, &chosen), "Trainer::step: gs_autotune");
    retunes_.push_back({step, reduction()});
  }
  gs_step_result r;
  check(gs_step(gpu_, GS_STEP_TRAIN | (profile ? GS_STEP_PROFILE : 0u), &r), "Trainer::step: gs_step");
  // A step whose pairs did not fit left the model alone: no pose or gain update either.
  if (!r.overflow && (pose || exposure || motion)) learn_corrections(frames, r, pose, exposure, motion);
  // Statistics: the views' sums (read_slot / set_view_stats), averaged over the views.
  const double lambda = lambda_at(step);
  ViewLosses mean;
  stats_.pairs = 0;
  for (uint32_t v = 0; v < k; ++v) {
    const ViewLosses l = view_losses(r.losses[v], cams[v].width, cams[v].height, lambda, ssim);
    mean.l1 += l.l1 / k;
    mean.psnr += l.psnr / k;
    mean.ssim += l.ssim / k;
    mean.loss += l.loss / k;
    stats_.pairs += r.pairs[v];
  }
  stats_.l1 = mean.l1;
  stats_.psnr = mean.psnr;
  stats_.ssim = mean.ssim;
  stats_.loss = mean.loss;
  stats_.tile_mismatch = r.tile_mismatch;
  if (r.overflow) ++stats_.overflow_steps;
  stats_.sh_degree = int(sh_degree_at(step));
  if (profile) {
    profile_.project = r.pass_ms[0];
    profile_.sort = r.pass_ms[1];
    profile_.rasterize = r.pass_ms[2];
    profile_.ssim = r.pass_ms[3];
    profile_.backward = r.pass_ms[4];
    profile_.optimize = r.pass_ms[5];
    profile_.valid = true;
  }
  frame_bytes_.assign(reinterpret_cast<const uint8_t*>(&fd[0]), reinterpret_cast<const uint8_t*>(&fd[0]) + sizeof(fd[0]));
  ++stats_.step;
  stats_.views += k;
  after_step();
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
  auto ema = [](double& avg, double v) { avg = avg == 0.0 ? v : 0.9 * avg + 0.1 * v; };
  ema(stats_.step_ms, ms);
  ema(stats_.timing.wall_ms, ms);
  ema(stats_.timing.gpu_ms, double(r.gpu_ms));
  ema(stats_.timing.batch, double(k));
}

void Trainer::step(bool profile) {
  std::vector<size_t> frames(options_.views_per_step);
  std::vector<std::array<float, 3>> bgs(options_.views_per_step);
  for (uint32_t v = 0; v < options_.views_per_step; ++v) next_view(frames[v], bgs[v].data());
  run_step(frames, bgs, profile);
}

void Trainer::step_on(size_t frame, const float background[3], bool profile) {
  if (frame >= dataset_.frames.size()) throw std::out_of_range("Trainer::step_on: no such frame");
  run_step({frame}, {{background[0], background[1], background[2]}}, profile);
}

uint32_t Trainer::steps(uint32_t count) {
  uint32_t done = 0;
  while (done < count && !finished()) {
    step();
    ++done;
  }
  return done;
}

void Trainer::after_step() {
  const uint32_t t = stats_.step;
  bool densified = false;
  if (t < options_.densify_until) {
    if (t > options_.densify_from && options_.densify_interval > 0 && t % options_.densify_interval == 0) {
      densify();  // gs_densify binds the new gaussians to their nodes
      densified = true;
      bound_at_ = t;
    }
    if (options_.opacity_reset_interval > 0 && t % options_.opacity_reset_interval == 0) reset_opacity();
  }
  // The gaussians drift away from their nodes: bind them again every 100 steps
  // (trainer.cpp:949-950).
  if (!nodes_.empty() && !densified && t >= bound_at_ + 100) bind_motion();
}

void Trainer::densify() {
  // The last step's frame, its prune thresholds refreshed for the current step.
  gs_frame_data f;
  std::memcpy(&f, frame_bytes_.data(), sizeof(f));
  const bool prune_big = options_.opacity_reset_interval > 0 && stats_.step > options_.opacity_reset_interval;
  f.densify0[3] = prune_big ? 0.1f * dataset_.camera_extent : 0.0f;
  f.densify1[0] = prune_big ? 20.0f : 0.0f;
  const uint32_t slots_before = stats_.slots;
  uint32_t counters[4];
  check(gs_densify(gpu_, &f, counters), "Trainer::densify: gs_densify");
  const uint32_t free_slots = counters[0], spawned = counters[1], pruned = counters[2];
  const uint32_t room = free_slots + (capacity_ - slots_before);
  const uint32_t placed = std::min(spawned, room);
  stats_.slots = counters[3];
  stats_.gaussians = stats_.gaussians - pruned + placed;
  stats_.spawned += placed;
  stats_.pruned += pruned;
  ++stats_.densify_events;
}

void Trainer::reset_opacity() {
  const float max_logit = std::log(0.01f / (1.0f - 0.01f));
  check(gs_reset_opacity(gpu_, max_logit), "Trainer::reset_opacity");
}


std::vector<uint8_t> Trainer::render(const Camera& camera, const float background[3]) {
  return render_with(camera, background, nullptr);
}

std::vector<uint8_t> Trainer::render_with(const Camera& camera, const float background[3],
                                          const std::vector<float>* moved) {
  gs_frame_data f;
  const bool moving = moved != nullptr && !nodes_.empty();
  detail::frame_geometry(f, camera, stats_.slots, sh_stride_, int(sh_degree_at(stats_.step)),
                         moving ? GS_FLAG_MOTION : 0u, background);
  if (moving) upload_motion(0, *moved);  // gs_render moves the subject by view 0's motion
  std::vector<uint8_t> out(size_t(camera.width) * camera.height * 4);
  check(gs_render(gpu_, &f, out.data()), "Trainer::render");
  return out;
}

std::vector<uint8_t> Trainer::render_view(size_t frame, const float background[3]) {
  if (!moves_subject()) return render_with(camera_for(frame), background, nullptr);
  const std::vector<float> table = motion_table(frame);
  return render_with(camera_for(frame), background, &table);
}

void Trainer::run_eval_view(const Camera& camera, size_t frame, const uint8_t* rgba, const float gain[3],
                            uint32_t flags, const std::vector<float>* moved, gs_step_result& r) {
  // A measurement renders forward only with SSIM; an alignment probe trains with only the
  // camera moving (pose gradient, the model untouched) on L1 (trainer.cpp:1180-1183, 1250).
  const float black[3] = {0.0f, 0.0f, 0.0f};
  const bool align = (flags & GS_FLAG_POSE_ONLY) != 0u;
  const bool moving = moved != nullptr && !nodes_.empty();
  gs_frame_data f;
  write_frame(f, camera, black, stats_.step, !align, options_.masked, flags | (moving ? GS_FLAG_MOTION : 0u), gain);
  if (rgba != nullptr) {  // another dataset's image, uploaded with the step
    check(gs_set_views(gpu_, 1, &f, &rgba), "Trainer::evaluate: gs_set_views");
  } else {
    const uint32_t image = uint32_t(frame);
    check(gs_set_views_dataset(gpu_, 1, &f, &image), "Trainer::evaluate: gs_set_views_dataset");
  }
  if (moving) upload_motion(0, *moved);
  check(gs_step(gpu_, align ? GS_STEP_TRAIN : 0u, &r), "Trainer::evaluate: gs_step");
}

EvalResult Trainer::evaluate() { return evaluate_views(dataset_, true); }

EvalResult Trainer::evaluate_at_rest(const Dataset& other) {
  for (const DatasetFrame& f : other.frames) {
    const Camera c = dataset_camera(other, f);
    if (f.holdout && f.rgba.size() != size_t(c.width) * c.height * 4)
      throw std::runtime_error("Trainer::evaluate_at_rest: frame " + f.name + " has the wrong image size");
  }
  return evaluate_views(other, false);
}

EvalResult Trainer::evaluate_views(const Dataset& ds, bool own) {
  // evaluate_views (trainer.cpp:1244-1292): the held-out views of this trainer's own
  // dataset (poses, gains and motions as trained) or of another (the subject at rest).
  EvalResult result;
  const bool align = options_.refine_poses && options_.eval_pose_steps > 0;
  double sums[5] = {0, 0, 0, 0, 0}, unaligned = 0.0;
  const bool moving = own && moves_subject();
  auto measure = [&](const Camera& cam, size_t i, const float gain[3], const std::vector<float>* moved,
                     double* psnr_out) {
    gs_step_result r;
    run_eval_view(cam, i, own ? nullptr : ds.frames[i].rgba.data(), gain, 0u, moved, r);
    const ViewLosses l = view_losses(r.losses[0], cam.width, cam.height, lambda_at(stats_.step), true);
    if (psnr_out) {
      *psnr_out += l.psnr;
      return;
    }
    sums[0] += l.psnr;
    sums[1] += l.l1;
    sums[2] += l.ssim;
    if (r.losses[0][7] > 0.0) {  // the head region's pixels
      sums[3] += -10.0 * std::log10(std::max(r.losses[0][6] / (3.0 * r.losses[0][7]), 1e-12));
      sums[4] += 1.0;
    }
  };
  for (size_t i = 0; i < ds.frames.size(); ++i) {
    if (!ds.frames[i].holdout) continue;
    float gain[3] = {1.0f, 1.0f, 1.0f};
    if (own) view_gain(i, gain);
    std::vector<float> table;
    if (moving) table = motion_table(i);
    const std::vector<float>* m = moving ? &table : nullptr;
    const Camera given = dataset_camera(ds, ds.frames[i]);
    Camera seen = given;
    if (align) {
      measure(given, i, gain, m, &unaligned);
      seen = align_view(given, i, own ? nullptr : ds.frames[i].rgba.data(), gain, m, own);
    }
    measure(seen, i, gain, m, nullptr);
    ++result.views;
  }
  if (result.views > 0) {
    result.psnr = sums[0] / result.views;
    result.l1 = sums[1] / result.views;
    result.ssim = sums[2] / result.views;
    result.head_views = uint32_t(sums[4]);
    result.head_psnr = sums[4] > 0.0 ? sums[3] / sums[4] : 0.0;
    result.aligned = align;
    result.psnr_unaligned = align ? unaligned / result.views : result.psnr;
  }
  return result;
}

SplatScene Trainer::export_scene() {
  gs_model_info info;
  check(gs_model_info_get(gpu_, &info), "Trainer::export_scene");
  std::vector<float> p(size_t(info.slots) * 16), s(size_t(info.slots) * sh_stride_);
  uint32_t slots = 0;
  check(gs_model_export(gpu_, p.data(), sh_stride_ ? s.data() : nullptr, info.slots, &slots),
        "Trainer::export_scene: gs_model_export");
  SplatScene scene;
  scene.convention = AxisConvention::RUB;
  uint32_t alive = 0;
  for (uint32_t i = 0; i < slots; ++i) alive += p[size_t(i) * 16 + 7] > 0.5f ? 1u : 0u;
  scene.resize(alive, options_.sh_degree);
  const int coeffs = sh_rest_coeffs(options_.sh_degree);
  uint32_t o = 0;
  for (uint32_t i = 0; i < slots; ++i) {
    const float* d = &p[size_t(i) * 16];
    if (d[7] < 0.5f) continue;
    for (int k = 0; k < 3; ++k) {
      scene.positions[size_t(o) * 3 + k] = d[k];
      scene.log_scales[size_t(o) * 3 + k] = d[4 + k];
      scene.sh_dc[size_t(o) * 3 + k] = d[12 + k];
    }
    scene.opacity_logits[o] = d[3];
    const float len = std::sqrt(d[8] * d[8] + d[9] * d[9] + d[10] * d[10] + d[11] * d[11]);
    for (int k = 0; k < 4; ++k) scene.rotations[size_t(o) * 4 + k] = len > 0.0f ? d[8 + k] / len : (k == 0 ? 1.0f : 0.0f);
    for (int j = 0; j < coeffs * 3; ++j) scene.sh_rest[size_t(o) * coeffs * 3 + j] = s[size_t(i) * sh_stride_ + j];
    ++o;
  }
  return scene;
}

Trainer::Gradients Trainer::first_step_gradients() {
  gs_model_info info;
  check(gs_model_info_get(gpu_, &info), "Trainer::first_step_gradients");
  Gradients g;
  g.params.resize(size_t(info.slots) * 16);
  g.sh.resize(size_t(info.slots) * sh_stride_);
  check(gs_model_moments(gpu_, g.params.data(), nullptr, sh_stride_ ? g.sh.data() : nullptr, nullptr),
        "Trainer::first_step_gradients: gs_model_moments");
  for (float& v : g.params) v /= (1.0f - kBeta1);
  for (float& v : g.sh) v /= (1.0f - kBeta1);
  return g;
}

Trainer::DebugSnapshot Trainer::debug_snapshot() {
  auto fetch = [&](gs_snapshot_kind kind, auto& out) {
    size_t bytes = 0;
    check(gs_snapshot(gpu_, 0, kind, nullptr, 0, &bytes), "Trainer::debug_snapshot");
    out.resize(bytes / sizeof(out[0]));
    if (bytes) check(gs_snapshot(gpu_, 0, kind, out.data(), bytes, &bytes), "Trainer::debug_snapshot");
  };
  DebugSnapshot d;
  fetch(GS_SNAP_PIXEL_COUNT, d.pixel_count);
  fetch(GS_SNAP_PIXEL_GRAD, d.pixel_grad);
  fetch(GS_SNAP_PROJECTED, d.projected);
  fetch(GS_SNAP_TILES, d.tiles);
  fetch(GS_SNAP_OFFSETS, d.offsets);
  gs_tuning t;
  check(gs_get_tuning(gpu_, &t), "Trainer::debug_snapshot");
  if (t.deterministic) {  // an atomic training step keeps neither per-pair gradients nor pair indices
    fetch(GS_SNAP_PAIR_GRADS, d.pair_grads);
    fetch(GS_SNAP_PAIR_TILE, d.pair_tile);
    fetch(GS_SNAP_RENDER_ORDER, d.render_order);
  }
  fetch(GS_SNAP_DEPTH_KEY, d.depth_key);
  return d;
}

}  // namespace gs
