// Camera pose and exposure refinement of gs::Trainer (engine/src/trainer.cpp:1164-1394,
// 1691-1771). The GPU step sums each view's pose gradient and its exposure-fit sums
// (gs_step_result.pose_grad / .fit); the corrections themselves are small host-side state
// per dataset frame:
//  - a pose correction [E | d] applied after the dataset's world -> camera [R | t], giving
//    [E R | E t + d], moved by Adam on the 6-vector (shift d, turn w) with the shift's rate
//    scaled by the camera extent and both decaying to lr_pose_final over the run;
//  - a log gain per channel, blended towards log(sum R P / sum R^2) of each trained view,
//    used centred on the trained views' mean and interpolated for views not trained on.
#include <algorithm>
#include <cmath>
#include <limits>

#include "gs/trainer.h"
#include "gs_cuda.h"

namespace gs {

namespace {

constexpr double kBeta1 = 0.9, kBeta2 = 0.999;  // trainer.cpp:68-69
constexpr double kPi = 3.14159265358979323846;

// exp([w]x) by Rodrigues' formula: I + sin(t)/t K + (1 - cos t)/t^2 K^2, K = [w]x, t = |w|
// (series limits below 1e-9).
void turn_matrix(const double w[3], double E[9]) {
  const double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2], t = std::sqrt(t2);
  const double a = t > 1e-9 ? std::sin(t) / t : 1.0;
  const double b = t > 1e-9 ? (1.0 - std::cos(t)) / t2 : 0.5;
  const double K[9] = {0.0, -w[2], w[1], w[2], 0.0, -w[0], -w[1], w[0], 0.0};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double k2 = 0.0;
      for (int i = 0; i < 3; ++i) k2 += K[r * 3 + i] * K[i * 3 + c];
      E[r * 3 + c] = (r == c ? 1.0 : 0.0) + a * K[r * 3 + c] + b * k2;
    }
}

// The turn vector of a rotation matrix (the inverse of turn_matrix for angles below pi).
void turn_vector(const float R[9], double w[3]) {
  const double t = std::acos(std::clamp(0.5 * (double(R[0]) + R[4] + R[8] - 1.0), -1.0, 1.0));
  const double s = std::sin(t);
  const double f = s > 1e-9 ? t / (2.0 * s) : 0.5;
  w[0] = f * (double(R[7]) - R[5]);
  w[1] = f * (double(R[2]) - R[6]);
  w[2] = f * (double(R[3]) - R[1]);
}

// Degrees turned by a rotation matrix.
double turn_degrees(const float R[9]) {
  return std::acos(std::clamp(0.5 * (double(R[0]) + R[4] + R[8] - 1.0), -1.0, 1.0)) * 180.0 / kPi;
}

}  // namespace

Camera Trainer::with_fix(Camera cam, const PoseFix& p) {
  if (p.updates == 0) return cam;
  float rot[9], t[3];
  for (int r = 0; r < 3; ++r) {
    t[r] = p.shift[r];
    for (int c = 0; c < 3; ++c) {
      rot[r * 3 + c] = 0.0f;
      for (int k = 0; k < 3; ++k) rot[r * 3 + c] += p.rotation[r * 3 + k] * cam.rotation[k * 3 + c];
      t[r] += p.rotation[r * 3 + c] * cam.translation[c];
    }
  }
  std::copy(rot, rot + 9, cam.rotation);
  std::copy(t, t + 3, cam.translation);
  // The centre: -R^T t.
  for (int c = 0; c < 3; ++c) cam.position[c] = -(rot[c] * t[0] + rot[3 + c] * t[1] + rot[6 + c] * t[2]);
  return cam;
}

Camera Trainer::camera_for(size_t frame) const {
  const Camera cam = dataset_camera(dataset_, dataset_.frames.at(frame));
  return frame < pose_fix_.size() ? with_fix(cam, pose_fix_[frame]) : cam;
}

void Trainer::apply_pose_step(PoseFix& p, const double step[6]) {
  // The step's [E | d] applied after the current correction: [R | s] <- [E R | E s + d].
  double E[9];
  turn_matrix(step + 3, E);
  float rot[9], shift[3];
  for (int r = 0; r < 3; ++r) {
    shift[r] = float(step[r]);
    for (int c = 0; c < 3; ++c) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += E[r * 3 + k] * p.rotation[k * 3 + c];
      rot[r * 3 + c] = float(v);
      shift[r] += float(E[r * 3 + c] * p.shift[c]);
    }
  }
  std::copy(rot, rot + 9, p.rotation);
  std::copy(shift, shift + 3, p.shift);
}

void Trainer::update_pose(const double grad[6], size_t frame) {
  // Adam on (shift, turn) with bias correction by the frame's own update count
  // (update_pose, trainer.cpp:1350-1368).
  std::copy(grad, grad + 6, last_pose_grad_);
  PoseFix& p = pose_fix_.at(frame);
  ++p.updates;
  const double c1 = 1.0 / (1.0 - std::pow(kBeta1, double(p.updates)));
  const double c2 = 1.0 / (1.0 - std::pow(kBeta2, double(p.updates)));
  const double t = options_.iterations > 0 ? std::min(1.0, double(stats_.step) / options_.iterations) : 1.0;
  const double decay = std::pow(double(std::max(options_.lr_pose_final, 1e-6f)), t);
  double step[6];
  for (int i = 0; i < 6; ++i) {
    p.m[i] = kBeta1 * p.m[i] + (1.0 - kBeta1) * grad[i];
    p.v[i] = kBeta2 * p.v[i] + (1.0 - kBeta2) * grad[i] * grad[i];
    const double lr =
        (i < 3 ? double(options_.lr_pose_shift) * dataset_.camera_extent : double(options_.lr_pose_turn)) * decay;
    step[i] = p.v[i] > 0.0 ? -lr * (p.m[i] * c1) / (std::sqrt(p.v[i] * c2) + 1e-30) : 0.0;
  }
  apply_pose_step(p, step);
}

Trainer::PoseFix Trainer::align_camera(const Camera& camera, size_t frame, const uint8_t* rgba, const float gain[3],
                                       const ViewMotion* motion, const PoseFix* start) {
  // align_camera (trainer.cpp:1164-1212): from the better of the given pose and `start`,
  // normalised gradient steps on the L1 loss that grow by 1.5 after a step that lowered it
  // and halve (from the best pose) after one that did not; turns count as the shift they
  // cause at the camera extent. The best pose seen is kept, so never worse than given.
  const double reach = dataset_.camera_extent;
  PoseFix best{};
  double best_loss = std::numeric_limits<double>::infinity(), best_grad[6] = {0, 0, 0, 0, 0, 0};
  auto try_fix = [&](const PoseFix& fix) {
    gs_step_result r;
    run_eval_view(with_fix(camera, fix), frame, rgba, gain, GS_FLAG_POSE_GRAD | GS_FLAG_POSE_ONLY, motion, r);
    const double loss = r.losses[0][3];
    if (!(loss < best_loss)) return false;
    best = fix;
    best_loss = loss;
    std::copy(r.pose_grad[0], r.pose_grad[0] + 6, best_grad);
    return true;
  };
  if (options_.eval_pose_steps == 0) return best;
  uint32_t renders = 0;
  try_fix(PoseFix{});
  ++renders;
  if (start && start->updates > 0 && renders < options_.eval_pose_steps) {
    try_fix(*start);
    ++renders;
  }
  double length = double(options_.eval_pose_step) * reach;
  for (; renders < options_.eval_pose_steps; ++renders) {
    double g[6], norm = 0.0;
    for (int c = 0; c < 6; ++c) {
      g[c] = c < 3 ? best_grad[c] : best_grad[c] / reach;
      norm += g[c] * g[c];
    }
    if (!(norm > 0.0)) break;
    norm = std::sqrt(norm);
    double step[6];
    for (int c = 0; c < 6; ++c) step[c] = -length * g[c] / norm / (c < 3 ? 1.0 : reach);
    PoseFix next = best;
    next.updates = std::max(next.updates, 1u);
    apply_pose_step(next, step);
    length *= try_fix(next) ? 1.5 : 0.5;
  }
  return best;
}

Trainer::PoseFix Trainer::neighbour_fix(size_t frame) const {
  // Between the corrections of the training views before and after it in the capture
  // (neighbour_fix, trainer.cpp:1214-1241): shifts and turn vectors interpolated linearly.
  size_t a = train_before_.at(frame), b = train_after_.at(frame);
  if (a != kNone && pose_fix_[a].updates == 0) a = kNone;
  if (b != kNone && pose_fix_[b].updates == 0) b = kNone;
  PoseFix out{};
  if (a == kNone && b == kNone) return out;
  const double t = a == kNone ? 1.0 : b == kNone ? 0.0 : double(frame - a) / double(b - a);
  double wa[3] = {0, 0, 0}, wb[3] = {0, 0, 0};
  if (a != kNone) turn_vector(pose_fix_[a].rotation, wa);
  if (b != kNone) turn_vector(pose_fix_[b].rotation, wb);
  if (a == kNone) std::copy(wb, wb + 3, wa);
  if (b == kNone) std::copy(wa, wa + 3, wb);
  double w[3];
  for (int c = 0; c < 3; ++c) {
    const double sa = a == kNone ? pose_fix_[b].shift[c] : pose_fix_[a].shift[c];
    const double sb = b == kNone ? pose_fix_[a].shift[c] : pose_fix_[b].shift[c];
    out.shift[c] = float(sa + (sb - sa) * t);
    w[c] = wa[c] + (wb[c] - wa[c]) * t;
  }
  double E[9];
  turn_matrix(w, E);
  for (int i = 0; i < 9; ++i) out.rotation[i] = float(E[i]);
  out.updates = 1;
  return out;
}

void Trainer::update_pose_stats() {
  double shift_sum = 0.0, turn_sum = 0.0, shift_max = 0.0, turn_max = 0.0;
  uint32_t n = 0, updates = 0;
  for (size_t i : train_frames_) {
    const PoseFix& p = pose_fix_[i];
    if (p.updates == 0) continue;
    const Camera a = dataset_camera(dataset_, dataset_.frames[i]), b = camera_for(i);
    double d2 = 0.0;
    for (int k = 0; k < 3; ++k) d2 += (double(b.position[k]) - a.position[k]) * (double(b.position[k]) - a.position[k]);
    const double shift = std::sqrt(d2), turn = turn_degrees(p.rotation);
    shift_sum += shift;
    turn_sum += turn;
    shift_max = std::max(shift_max, shift);
    turn_max = std::max(turn_max, turn);
    updates += p.updates;
    ++n;
  }
  stats_.pose_shift_mean = n ? shift_sum / n : 0.0;
  stats_.pose_turn_mean = n ? turn_sum / n : 0.0;
  stats_.pose_shift_max = shift_max;
  stats_.pose_turn_max = turn_max;
  stats_.pose_updates = updates;
}

void Trainer::update_exposure(const double fit[8], size_t frame) {
  // The gain per channel that best maps the model's colour to the photo where both are
  // opaque, sum R P / sum R^2, clamped to [1/4, 4]; its log blended in at exposure_rate
  // (the first measurement taken as is). Skipped with under 500 such pixels
  // (update_exposure, trainer.cpp:1697-1711).
  if (fit[3] < 500.0) return;
  std::array<double, 3>& g = gain_log_.at(frame);
  const double rate = gain_updates_[frame] == 0 ? 1.0 : std::clamp(double(options_.exposure_rate), 0.0, 1.0);
  for (int c = 0; c < 3; ++c) {
    if (!(fit[c] > 1e-9)) continue;
    const double fitted = std::log(std::clamp(fit[4 + c] / fit[c], 0.25, 4.0));
    g[c] = (1.0 - rate) * g[c] + rate * fitted;
  }
  ++gain_updates_[frame];
}

std::array<float, 3> Trainer::exposure_gain(size_t frame) const {
  // Only the gains' ratios are fixed by the photos, so they are used divided by their
  // geometric mean over the measured training views (exposure_gain, trainer.cpp:1713-1744).
  std::array<float, 3> out = {1.0f, 1.0f, 1.0f};
  if (frame >= gain_log_.size()) return out;
  double mean[3] = {0, 0, 0};
  size_t views = 0;
  for (size_t v : train_frames_) {
    if (gain_updates_[v] == 0) continue;
    for (int c = 0; c < 3; ++c) mean[c] += gain_log_[v][c];
    ++views;
  }
  if (views == 0) return out;
  for (double& m : mean) m /= double(views);
  if (gain_updates_[frame] > 0) {
    for (int c = 0; c < 3; ++c) out[c] = float(std::exp(gain_log_[frame][c] - mean[c]));
    return out;
  }
  // Not measured: between the measured training views before and after it in the capture.
  size_t a = train_before_[frame], b = train_after_[frame];
  if (a != kNone && gain_updates_[a] == 0) a = kNone;
  if (b != kNone && gain_updates_[b] == 0) b = kNone;
  if (a == kNone && b == kNone) return out;
  const double t = a == kNone ? 1.0 : b == kNone ? 0.0 : double(frame - a) / double(b - a);
  for (int c = 0; c < 3; ++c) {
    const double la = a == kNone ? gain_log_[b][c] : gain_log_[a][c];
    const double lb = b == kNone ? gain_log_[a][c] : gain_log_[b][c];
    out[c] = float(std::exp(la + (lb - la) * t - mean[c]));
  }
  return out;
}

void Trainer::view_gain(size_t frame, float gain[3]) const {
  const std::array<float, 3> g = exposure_gain(frame);
  std::copy(g.begin(), g.end(), gain);
}

void Trainer::update_exposure_stats() {
  // The spread of the trained views' gains: 5th / 95th percentile luminance gain and the
  // standard deviation of the tint (red + blue) / 2 / green (trainer.cpp:1751-1771).
  std::vector<double> lum, tint;
  uint32_t updates = 0;
  for (size_t v : train_frames_) {
    if (gain_updates_[v] == 0) continue;
    updates += gain_updates_[v];
    const std::array<float, 3> g = exposure_gain(v);
    lum.push_back(0.299 * g[0] + 0.587 * g[1] + 0.114 * g[2]);
    tint.push_back(0.5 * (double(g[0]) + g[2]) / std::max(double(g[1]), 1e-6));
  }
  stats_.exposure_updates = updates;
  if (lum.empty()) return;
  std::sort(lum.begin(), lum.end());
  stats_.exposure_low = lum[size_t(0.05 * double(lum.size() - 1))];
  stats_.exposure_high = lum[size_t(0.95 * double(lum.size() - 1) + 0.5)];
  double mean = 0.0, sq = 0.0;
  for (double x : tint) mean += x;
  mean /= double(tint.size());
  for (double x : tint) sq += (x - mean) * (x - mean);
  stats_.exposure_tint = tint.size() > 1 ? std::sqrt(sq / double(tint.size() - 1)) : 0.0;
}

}  // namespace gs
