// Subject motion of gs::Trainer (SC-GS; engine/src/trainer.cpp:1398-1690, trainer.h:83-117).
// The GPU moves the gaussians with each view's node motions and sums the image loss's
// gradient per node (gs_set_view_motion, GS_FLAG_MOTION_GRAD, gs_motion_gradient); the
// host keeps the nodes, every view's motions and their Adam state, and adds the penalties
// that keep the motions small, rigid between neighbouring nodes, smooth between
// neighbouring views and centred on the rest pose.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <random>

#include "gs/trainer.h"
#include "gs_cuda.h"

namespace gs {

namespace {

constexpr double kBeta1 = 0.9, kBeta2 = 0.999;  // trainer.cpp:68-69
constexpr double kPi = 3.14159265358979323846;

// exp([w]x) by Rodrigues' formula (series limits below 1e-9).
void turn_matrix(const double w[3], double E[9]) {
  const double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2], t = std::sqrt(t2);
  const double a = t > 1e-9 ? std::sin(t) / t : 1.0;
  const double b = t > 1e-9 ? (1.0 - std::cos(t)) / t2 : 0.5;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) E[r * 3 + c] = (r == c ? 1.0 - b * t2 : 0.0) + b * w[r] * w[c];
  E[1] -= a * w[2];
  E[2] += a * w[1];
  E[3] += a * w[2];
  E[5] -= a * w[0];
  E[6] -= a * w[1];
  E[7] += a * w[0];
}

float dist2(const std::array<float, 3>& a, const std::array<float, 3>& b) {
  const float x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
  return x * x + y * y + z * z;
}

}  // namespace

void Trainer::place_nodes(const SplatScene& initial) {
  // k-means over up to 20000 of the initial gaussians (k-means++ seeds, 15 Lloyd
  // iterations): the nodes spread over the subject like its surface. Its own generator, so
  // the view order is the same as without motion.
  if (initial.count == 0) return;
  const uint32_t stride = std::max(1u, initial.count / 20000u);
  std::vector<std::array<float, 3>> pts;
  for (uint32_t i = 0; i < initial.count; i += stride)
    pts.push_back({initial.positions[i * 3], initial.positions[i * 3 + 1], initial.positions[i * 3 + 2]});
  const size_t k_count = std::min<size_t>({options_.motion_nodes, size_t(GS_MAX_MOTION_NODES), pts.size()});
  if (k_count == 0) return;
  std::mt19937 rng(options_.seed * 2654435761u + 97u);
  std::vector<std::array<float, 3>> centres{pts[std::uniform_int_distribution<size_t>(0, pts.size() - 1)(rng)]};
  std::vector<float> nearest(pts.size(), std::numeric_limits<float>::max());
  while (centres.size() < k_count) {
    double total = 0.0;
    for (size_t i = 0; i < pts.size(); ++i) {
      nearest[i] = std::min(nearest[i], dist2(pts[i], centres.back()));
      total += nearest[i];
    }
    // The next seed drawn with probability proportional to the squared distance.
    double pick = std::uniform_real_distribution<double>(0.0, total)(rng);
    size_t chosen = pts.size() - 1;
    for (size_t i = 0; i < pts.size(); ++i) {
      pick -= nearest[i];
      if (pick <= 0.0) {
        chosen = i;
        break;
      }
    }
    centres.push_back(pts[chosen]);
  }
  for (int iteration = 0; iteration < 15; ++iteration) {
    std::vector<std::array<double, 4>> sum(k_count, {0, 0, 0, 0});
    for (const auto& p : pts) {
      size_t owner = 0;
      float best = std::numeric_limits<float>::max();
      for (size_t k = 0; k < k_count; ++k) {
        const float d = dist2(p, centres[k]);
        if (d < best) {
          best = d;
          owner = k;
        }
      }
      for (int c = 0; c < 3; ++c) sum[owner][c] += p[c];
      sum[owner][3] += 1.0;
    }
    for (size_t k = 0; k < k_count; ++k)
      if (sum[k][3] > 0.0)  // an empty cluster keeps its place
        for (int c = 0; c < 3; ++c) centres[k][c] = float(sum[k][c] / sum[k][3]);
  }
  // Radius: the mean distance to the 3 nearest other nodes; neighbours: the 6 nearest.
  nodes_.assign(k_count, MotionNode{});
  node_neighbors_.assign(k_count, {});
  std::vector<float> radii;
  for (size_t k = 0; k < k_count; ++k) {
    std::vector<std::pair<float, uint32_t>> others;
    for (size_t j = 0; j < k_count; ++j)
      if (j != k) others.emplace_back(std::sqrt(dist2(centres[k], centres[j])), uint32_t(j));
    std::sort(others.begin(), others.end());
    const size_t near = std::min<size_t>(3, others.size());
    double r = 0.0;
    for (size_t j = 0; j < near; ++j) r += others[j].first;
    float radius = near > 0 ? float(r / double(near)) : 0.0f;
    if (!(radius > 1e-4f)) radius = std::max(0.05f * dataset_.camera_extent, 1e-3f);
    for (size_t j = 0; j < std::min<size_t>(6, others.size()); ++j) node_neighbors_[k].push_back(others[j].second);
    for (int c = 0; c < 3; ++c) nodes_[k].position[c] = centres[k][c];
    nodes_[k].radius = radius;
    radii.push_back(radius);
  }
  std::nth_element(radii.begin(), radii.begin() + radii.size() / 2, radii.end());
  node_spacing_ = radii[radii.size() / 2];
  motion_.assign(dataset_.frames.size(), ViewMotion(k_count));
  motion_updates_.assign(dataset_.frames.size(), 0u);
  stats_.motion_nodes = uint32_t(k_count);
  std::vector<float> nodes4(k_count * 4);
  for (size_t k = 0; k < k_count; ++k) {
    for (int c = 0; c < 3; ++c) nodes4[k * 4 + c] = nodes_[k].position[c];
    nodes4[k * 4 + 3] = 1.0f / (2.0f * nodes_[k].radius * nodes_[k].radius);
  }
  check(gs_motion_nodes(gpu_, uint32_t(k_count), nodes4.data()), "Trainer: gs_motion_nodes");
  bound_at_ = stats_.step;
}

void Trainer::bind_motion() {
  if (nodes_.empty()) return;
  check(gs_motion_bind(gpu_), "Trainer: gs_motion_bind");
  bound_at_ = stats_.step;
}

bool Trainer::uses_motion() const {
  return std::any_of(motion_updates_.begin(), motion_updates_.end(), [](uint32_t u) { return u > 0; });
}

Trainer::ViewMotion Trainer::view_motion(size_t frame) const {
  if (motion_updates_.at(frame) > 0) return motion_[frame];
  // Not trained: between the trained views before and after it in the capture (the
  // subject moves smoothly), turn vectors and shifts interpolated linearly.
  ViewMotion out(nodes_.size());
  size_t a = train_before_[frame], b = train_after_[frame];
  if (a != kNone && motion_updates_[a] == 0) a = kNone;
  if (b != kNone && motion_updates_[b] == 0) b = kNone;
  if (a == kNone && b == kNone) return out;
  const double t = a == kNone ? 1.0 : b == kNone ? 0.0 : double(frame - a) / double(b - a);
  const ViewMotion& ma = motion_[a == kNone ? b : a];
  const ViewMotion& mb = motion_[b == kNone ? a : b];
  for (size_t k = 0; k < nodes_.size(); ++k)
    for (int c = 0; c < 3; ++c) {
      out[k].turn[c] = float(ma[k].turn[c] + (double(mb[k].turn[c]) - ma[k].turn[c]) * t);
      out[k].shift[c] = float(ma[k].shift[c] + (double(mb[k].shift[c]) - ma[k].shift[c]) * t);
    }
  return out;
}

void Trainer::start_motion(size_t frame) {
  if (motion_updates_.at(frame) > 0) return;
  const ViewMotion guess = view_motion(frame);
  for (size_t k = 0; k < nodes_.size(); ++k) {
    std::copy(guess[k].turn, guess[k].turn + 3, motion_[frame][k].turn);
    std::copy(guess[k].shift, guess[k].shift + 3, motion_[frame][k].shift);
  }
}

void Trainer::set_motion_table(uint32_t view, const ViewMotion& motion) {
  // Per node: [R | b] with R = exp([turn]x), c = n + shift, b = c - R n; the turn; c.
  std::vector<float> table(nodes_.size() * 20, 0.0f);
  for (size_t k = 0; k < nodes_.size(); ++k) {
    const NodeMotion& m = motion[k];
    const double w[3] = {m.turn[0], m.turn[1], m.turn[2]};
    double R[9];
    turn_matrix(w, R);
    const float* n = nodes_[k].position;
    float* o = &table[k * 20];
    for (int r = 0; r < 3; ++r) {
      const double c = double(n[r]) + m.shift[r];
      double b = c;
      for (int j = 0; j < 3; ++j) {
        o[r * 4 + j] = float(R[r * 3 + j]);
        b -= R[r * 3 + j] * n[j];
      }
      o[r * 4 + 3] = float(b);
      o[12 + r] = m.turn[r];
      o[16 + r] = float(c);
    }
  }
  check(gs_set_view_motion(gpu_, view, table.data()), "Trainer: gs_set_view_motion");
}

void Trainer::update_motion(const double* image_grad, size_t frame) {
  // The image loss's gradient, then the penalties', then Adam with one second moment per
  // vector (shift, turn), so a step keeps the gradient's direction (update_motion,
  // trainer.cpp:1528-1634).
  const size_t K = nodes_.size();
  ViewMotion& m = motion_.at(frame);
  std::vector<double> grad(image_grad, image_grad + K * 6);
  last_motion_grad_ = grad;
  const double inv_s2 = 1.0 / (double(node_spacing_) * node_spacing_);
  const double decay = options_.motion_decay, rigid = options_.motion_rigidity;
  const double smooth = options_.motion_smoothness, centre = options_.motion_center;
  // Small: decay (|shift|^2 / s^2 + |turn|^2).
  for (size_t k = 0; k < K; ++k)
    for (int c = 0; c < 3; ++c) {
      grad[k * 6 + c] += 2.0 * decay * m[k].shift[c] * inv_s2;
      grad[k * 6 + 3 + c] += 2.0 * decay * m[k].turn[c];
    }
  if (rigid > 0.0) {
    // As rigid as possible: neighbour j should land where node k's motion takes it,
    // e = (n_j + s_j) - (n_k + s_k) - R_k (n_j - n_k); a turn u of R_k changes e by (R_k d) x u.
    const double f = 2.0 * rigid * inv_s2;
    for (size_t k = 0; k < K; ++k) {
      const double w[3] = {m[k].turn[0], m[k].turn[1], m[k].turn[2]};
      double R[9];
      turn_matrix(w, R);
      for (uint32_t j : node_neighbors_[k]) {
        double d[3], Rd[3], e[3];
        for (int c = 0; c < 3; ++c) d[c] = double(nodes_[j].position[c]) - nodes_[k].position[c];
        for (int r = 0; r < 3; ++r) {
          Rd[r] = R[r * 3] * d[0] + R[r * 3 + 1] * d[1] + R[r * 3 + 2] * d[2];
          e[r] = d[r] + m[j].shift[r] - m[k].shift[r] - Rd[r];
        }
        for (int c = 0; c < 3; ++c) {
          grad[j * 6 + c] += f * e[c];
          grad[k * 6 + c] -= f * e[c];
        }
        grad[k * 6 + 3] += f * (e[1] * Rd[2] - e[2] * Rd[1]);
        grad[k * 6 + 4] += f * (e[2] * Rd[0] - e[0] * Rd[2]);
        grad[k * 6 + 5] += f * (e[0] * Rd[1] - e[1] * Rd[0]);
      }
    }
  }
  if (centre > 0.0) {
    // Each node's mean motion over the trained views (this one included) pulled to zero.
    std::vector<double> mean(K * 6, 0.0);
    double views = 0.0;
    for (size_t f : train_frames_) {
      if (motion_updates_[f] == 0 && f != frame) continue;
      views += 1.0;
      for (size_t k = 0; k < K; ++k)
        for (int c = 0; c < 3; ++c) {
          mean[k * 6 + c] += motion_[f][k].shift[c];
          mean[k * 6 + 3 + c] += motion_[f][k].turn[c];
        }
    }
    const double f = 2.0 * centre / std::max(views, 1.0);
    for (size_t k = 0; k < K; ++k)
      for (int c = 0; c < 3; ++c) {
        grad[k * 6 + c] += f * mean[k * 6 + c] * inv_s2;
        grad[k * 6 + 3 + c] += f * mean[k * 6 + 3 + c];
      }
  }
  if (smooth > 0.0) {
    // Alike between the trained views before and after it in the capture.
    for (size_t other : {train_before_[frame], train_after_[frame]}) {
      if (other == kNone || motion_updates_[other] == 0) continue;
      for (size_t k = 0; k < K; ++k)
        for (int c = 0; c < 3; ++c) {
          grad[k * 6 + c] += 2.0 * smooth * (double(m[k].shift[c]) - motion_[other][k].shift[c]) * inv_s2;
          grad[k * 6 + 3 + c] += 2.0 * smooth * (double(m[k].turn[c]) - motion_[other][k].turn[c]);
        }
    }
  }
  const uint32_t n = ++motion_updates_[frame];
  const double c1 = 1.0 / (1.0 - std::pow(kBeta1, double(n)));
  const double c2 = 1.0 / (1.0 - std::pow(kBeta2, double(n)));
  const double t = options_.iterations > 0 ? std::min(1.0, double(stats_.step) / options_.iterations) : 1.0;
  const double fade = std::pow(double(std::max(options_.lr_motion_final, 1e-6f)), t);
  const double lr[2] = {double(options_.lr_motion_shift) * dataset_.camera_extent * fade,
                        double(options_.lr_motion_turn) * fade};
  for (size_t k = 0; k < K; ++k) {
    NodeMotion& node = m[k];
    for (int part = 0; part < 2; ++part) {
      double sq = 0.0;
      for (int c = 0; c < 3; ++c) {
        const double g = grad[k * 6 + part * 3 + c];
        node.m[part * 3 + c] = kBeta1 * node.m[part * 3 + c] + (1.0 - kBeta1) * g;
        sq += g * g;
      }
      node.v[part] = kBeta2 * node.v[part] + (1.0 - kBeta2) * sq / 3.0;
      if (!(node.v[part] > 0.0)) continue;
      const double denom = std::sqrt(node.v[part] * c2) + 1e-30;
      float* value = part == 0 ? node.shift : node.turn;
      for (int c = 0; c < 3; ++c) value[c] -= float(lr[part] * node.m[part * 3 + c] * c1 / denom);
    }
  }
}

void Trainer::update_motion_stats() {
  double shift_sum = 0.0, turn_sum = 0.0, shift_max = 0.0, turn_max = 0.0;
  size_t n = 0;
  uint32_t updates = 0;
  for (size_t f : train_frames_) {
    if (motion_updates_[f] == 0) continue;
    updates += motion_updates_[f];
    for (const NodeMotion& m : motion_[f]) {
      const double shift = std::sqrt(double(m.shift[0]) * m.shift[0] + double(m.shift[1]) * m.shift[1] +
                                     double(m.shift[2]) * m.shift[2]);
      const double turn = std::sqrt(double(m.turn[0]) * m.turn[0] + double(m.turn[1]) * m.turn[1] +
                                    double(m.turn[2]) * m.turn[2]) * 180.0 / kPi;
      shift_sum += shift;
      turn_sum += turn;
      shift_max = std::max(shift_max, shift);
      turn_max = std::max(turn_max, turn);
      ++n;
    }
  }
  stats_.motion_shift_mean = n ? shift_sum / double(n) : 0.0;
  stats_.motion_turn_mean = n ? turn_sum / double(n) : 0.0;
  stats_.motion_shift_max = shift_max;
  stats_.motion_turn_max = turn_max;
  stats_.motion_updates = updates;
}

void Trainer::node_motion(size_t frame, uint32_t node, float turn[3], float shift[3]) const {
  const NodeMotion& m = motion_.at(frame).at(node);
  std::copy(m.turn, m.turn + 3, turn);
  std::copy(m.shift, m.shift + 3, shift);
}

void Trainer::set_node_motion(size_t frame, uint32_t node, const float turn[3], const float shift[3]) {
  NodeMotion& m = motion_.at(frame).at(node);
  std::copy(turn, turn + 3, m.turn);
  std::copy(shift, shift + 3, m.shift);
  if (motion_updates_[frame] == 0) motion_updates_[frame] = 1;  // counts as trained: used as is
}

Trainer::MotionBinding Trainer::motion_binding() {
  MotionBinding b;
  if (nodes_.empty() || stats_.slots == 0) return b;
  size_t bytes = 0;
  check(gs_snapshot(gpu_, 0, GS_SNAP_MOTION_BIND, nullptr, 0, &bytes), "Trainer::motion_binding");
  std::vector<uint32_t> raw(bytes / 4);
  check(gs_snapshot(gpu_, 0, GS_SNAP_MOTION_BIND, raw.data(), bytes, &bytes), "Trainer::motion_binding");
  const size_t slots = raw.size() / 8;
  b.nodes.resize(slots * 4);
  b.weights.resize(slots * 4);
  for (size_t i = 0; i < slots; ++i)
    for (int j = 0; j < 4; ++j) {
      b.nodes[i * 4 + j] = raw[i * 8 + j];
      std::memcpy(&b.weights[i * 4 + j], &raw[i * 8 + 4 + j], 4);
    }
  return b;
}

}  // namespace gs
