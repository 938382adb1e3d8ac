// gs::Trainer's per-view corrections: camera pose refinement, exposure gains and subject
// motion, over the state of refinement.h and node_rig.h. The GPU step supplies, per view,
// the pose gradient (GS_FLAG_POSE_GRAD), the exposure fit sums and, with
// GS_FLAG_MOTION_GRAD, the image loss's gradient per motion node; the learning happens
// here, between steps. The reference's features these follow: pose refinement
// (trainer.h:69-81), exposure refinement (trainer.h:98-103) and subject motion
// (trainer.h:83-117), with their options and statistics.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "corrections.h"
#include "gs_cuda.h"

namespace gs {

double Trainer::rate_fade(float final_fraction) const {
  const double t = options_.iterations > 0 ? std::min(1.0, double(stats_.step) / options_.iterations) : 1.0;
  return std::pow(double(std::max(final_fraction, 1e-6f)), t);
}

Camera Trainer::camera_for(size_t frame) const {
  const Camera base = dataset_camera(dataset_, dataset_.frames.at(frame));
  return fix_->poses.learned(frame) ? fix_->poses.fix(frame).apply(base) : base;
}

void Trainer::view_gain(size_t frame, float gain[3]) const {
  const std::array<float, 3> g = fix_->gains.gains(frame, fix_->order);
  std::copy(g.begin(), g.end(), gain);
}

void Trainer::learn_corrections(const std::vector<size_t>& frames, const gs_step_result& r, bool pose, bool exposure,
                                bool motion) {
  const double extent = dataset_.camera_extent;
  const double pose_fade = rate_fade(options_.lr_pose_final), motion_fade = rate_fade(options_.lr_motion_final);
  refine::RigEnergy energy;
  energy.decay = options_.motion_decay;
  energy.rigidity = options_.motion_rigidity;
  energy.smoothness = options_.motion_smoothness;
  energy.centring = options_.motion_center;
  std::vector<double> node_grad(fix_->rig.size() * 6);
  for (size_t v = 0; v < frames.size(); ++v) {
    if (pose) {
      std::copy(r.pose_grad[v], r.pose_grad[v] + 6, last_pose_grad_);
      fix_->poses.learn(frames[v], r.pose_grad[v], options_.lr_pose_shift * extent * pose_fade,
                        options_.lr_pose_turn * pose_fade);
    }
    if (exposure) fix_->gains.observe(frames[v], r.fit[v], options_.exposure_rate);
    if (motion) {
      check(gs_motion_gradient(gpu_, uint32_t(v), node_grad.data(), uint32_t(fix_->rig.size())),
            "Trainer::step: gs_motion_gradient");
      last_motion_grad_ = node_grad;
      fix_->rig.learn(frames[v], node_grad.data(), energy, options_.lr_motion_shift * extent * motion_fade,
                      options_.lr_motion_turn * motion_fade, fix_->order);
    }
  }
  if (pose) {
    const refine::PoseTable::Spread s = fix_->poses.spread(
        train_frames_, [&](size_t f) { return dataset_camera(dataset_, dataset_.frames[f]); });
    stats_.pose_shift_mean = s.shift_mean;
    stats_.pose_shift_max = s.shift_max;
    stats_.pose_turn_mean = s.turn_mean;
    stats_.pose_turn_max = s.turn_max;
    stats_.pose_updates = s.updates;
  }
  if (exposure) {
    const refine::GainTable::Spread s = fix_->gains.spread(fix_->order);
    stats_.exposure_low = s.low;
    stats_.exposure_high = s.high;
    stats_.exposure_tint = s.tint;
    stats_.exposure_updates = s.updates;
  }
  if (motion) {
    const refine::NodeRig::Spread s = fix_->rig.spread(train_frames_);
    stats_.motion_shift_mean = s.shift_mean;
    stats_.motion_shift_max = s.shift_max;
    stats_.motion_turn_mean = s.turn_mean;
    stats_.motion_turn_max = s.turn_max;
    stats_.motion_updates = s.updates;
  }
}

Camera Trainer::align_view(const Camera& given, size_t frame, const uint8_t* rgba, const float gain[3],
                           const std::vector<float>* moved, bool own) {
  // From the dataset's pose and (own dataset) the frame's estimate: its own correction if it
  // was aligned before, else the blend of its trained neighbours'. Alignment probes move
  // only the camera, on L1 (GS_FLAG_POSE_ONLY skips the model's update).
  std::vector<refine::RigidFix> starts{refine::RigidFix{}};
  if (own) starts.push_back(fix_->poses.estimate(frame, fix_->order));
  auto probe = [&](const refine::RigidFix& fix, double& loss, double grad[6]) {
    gs_step_result r;
    run_eval_view(fix.apply(given), frame, rgba, gain, GS_FLAG_POSE_GRAD | GS_FLAG_POSE_ONLY, moved, r);
    loss = r.losses[0][3];
    std::copy(r.pose_grad[0], r.pose_grad[0] + 6, grad);
    return std::isfinite(loss);
  };
  const double reach = dataset_.camera_extent;
  const refine::RigidFix fix =
      refine::align(probe, starts, options_.eval_pose_steps, double(options_.eval_pose_step) * reach, reach);
  if (own) fix_->poses.assign(frame, fix);
  return fix.apply(given);
}

// ---- subject motion ----

void Trainer::build_rig(const SplatScene& initial) {
  const size_t count = std::min<size_t>(options_.motion_nodes, GS_MAX_MOTION_NODES);
  const float fallback = std::max(0.05f * dataset_.camera_extent, 1e-3f);
  fix_->rig.place(initial.positions, count, dataset_.frames.size(), fallback);
  nodes_.clear();
  if (fix_->rig.empty()) return;
  std::vector<float> rest;  // position, 1 / (2 r^2) per node
  for (const refine::NodeRig::Node& n : fix_->rig.nodes()) {
    nodes_.push_back({{n.at[0], n.at[1], n.at[2]}, n.radius});
    rest.insert(rest.end(), {n.at[0], n.at[1], n.at[2], 1.0f / (2.0f * n.radius * n.radius)});
  }
  stats_.motion_nodes = uint32_t(nodes_.size());
  check(gs_motion_nodes(gpu_, uint32_t(nodes_.size()), rest.data()), "Trainer: gs_motion_nodes");
  bound_at_ = stats_.step;
}

void Trainer::bind_motion() {
  if (nodes_.empty()) return;
  check(gs_motion_bind(gpu_), "Trainer: gs_motion_bind");
  bound_at_ = stats_.step;
}

bool Trainer::refines_motion_at(uint32_t step) const { return !nodes_.empty() && step >= options_.motion_from; }

bool Trainer::moves_subject() const {
  for (size_t f = 0; f < dataset_.frames.size() && !nodes_.empty(); ++f)
    if (fix_->rig.learned(f)) return true;
  return false;
}

std::vector<float> Trainer::motion_table(size_t frame) const {
  return fix_->rig.table(fix_->rig.estimate(frame, fix_->order));
}

void Trainer::upload_motion(uint32_t view, const std::vector<float>& table) {
  check(gs_set_view_motion(gpu_, view, table.data()), "Trainer: gs_set_view_motion");
}

void Trainer::node_motion(size_t frame, uint32_t node, float turn[3], float shift[3]) const {
  const refine::NodeMotion& m = fix_->rig.pose(frame).at(node);
  for (int c = 0; c < 3; ++c) {
    turn[c] = float(m.turn[c]);
    shift[c] = float(m.shift[c]);
  }
}

void Trainer::set_node_motion(size_t frame, uint32_t node, const float turn[3], const float shift[3]) {
  fix_->rig.set(frame, node, {turn[0], turn[1], turn[2]}, {shift[0], shift[1], shift[2]});
}

Trainer::MotionBinding Trainer::motion_binding() {
  // GS_SNAP_MOTION_BIND: per slot 4 node indices, then their 4 weights as float bits.
  MotionBinding out;
  if (nodes_.empty() || stats_.slots == 0) return out;
  size_t bytes = 0;
  check(gs_snapshot(gpu_, 0, GS_SNAP_MOTION_BIND, nullptr, 0, &bytes), "Trainer::motion_binding");
  std::vector<uint32_t> words(bytes / sizeof(uint32_t));
  check(gs_snapshot(gpu_, 0, GS_SNAP_MOTION_BIND, words.data(), bytes, &bytes), "Trainer::motion_binding");
  const size_t slots = words.size() / 8;
  out.nodes.reserve(slots * 4);
  out.weights.reserve(slots * 4);
  for (size_t i = 0; i < slots; ++i) {
    const uint32_t* w = &words[i * 8];
    out.nodes.insert(out.nodes.end(), w, w + 4);
    for (int j = 0; j < 4; ++j) {
      float f;
      std::memcpy(&f, &w[4 + j], sizeof(f));
      out.weights.push_back(f);
    }
  }
  return out;
}

}  // namespace gs
