// Control-node rig of subject motion (node_rig.h).
#include "node_rig.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace gs::refine {

namespace {

constexpr double kPi = 3.14159265358979323846;

using P3 = std::array<float, 3>;

float sq_dist(const P3& a, const P3& b) {
  const float x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
  return x * x + y * y + z * z;
}

double length(const Vec3& v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

Vec3 cross(const Vec3& a, const Vec3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}

// The index of the nearest of `centres` to p.
size_t nearest_of(const P3& p, const std::vector<P3>& centres) {
  size_t best = 0;
  float d = std::numeric_limits<float>::max();
  for (size_t k = 0; k < centres.size(); ++k) {
    const float e = sq_dist(p, centres[k]);
    if (e < d) {
      d = e;
      best = k;
    }
  }
  return best;
}

}  // namespace

void NodeRig::place(const std::vector<float>& xyz, size_t count, size_t frames, float fallback) {
  nodes_.clear();
  links_.clear();
  views_.clear();
  const size_t total = xyz.size() / 3;
  if (total == 0 || count == 0) return;
  const size_t every = (total + 19999) / 20000;
  std::vector<P3> pts;
  for (size_t i = 0; i < total; i += every) pts.push_back({xyz[i * 3], xyz[i * 3 + 1], xyz[i * 3 + 2]});
  const size_t k_count = std::min(count, pts.size());

  // Farthest-point seeds: from the point nearest the centroid, each next seed is the point
  // farthest from all seeds so far.
  P3 mean{0.0f, 0.0f, 0.0f};
  for (const P3& p : pts)
    for (int c = 0; c < 3; ++c) mean[c] += p[c] / float(pts.size());
  std::vector<P3> centres{pts[nearest_of(mean, pts)]};
  std::vector<float> gap(pts.size());
  for (size_t i = 0; i < pts.size(); ++i) gap[i] = sq_dist(pts[i], centres[0]);
  while (centres.size() < k_count) {
    const size_t far = size_t(std::max_element(gap.begin(), gap.end()) - gap.begin());
    centres.push_back(pts[far]);
    for (size_t i = 0; i < pts.size(); ++i) gap[i] = std::min(gap[i], sq_dist(pts[i], centres.back()));
  }
  // Lloyd refinement until the assignment settles.
  std::vector<size_t> owner(pts.size(), k_count);
  for (int round = 0; round < 25; ++round) {
    bool changed = false;
    std::vector<std::array<double, 3>> sum(k_count, {0.0, 0.0, 0.0});
    std::vector<size_t> members(k_count, 0);
    for (size_t i = 0; i < pts.size(); ++i) {
      const size_t k = nearest_of(pts[i], centres);
      changed = changed || k != owner[i];
      owner[i] = k;
      for (int c = 0; c < 3; ++c) sum[k][c] += pts[i][c];
      ++members[k];
    }
    if (!changed) break;
    for (size_t k = 0; k < k_count; ++k)
      if (members[k] > 0)
        for (int c = 0; c < 3; ++c) centres[k][c] = float(sum[k][c] / double(members[k]));
  }

  // Radii and links from the distances between nodes.
  nodes_.resize(k_count);
  links_.assign(k_count, {});
  std::vector<float> radii(k_count);
  for (size_t k = 0; k < k_count; ++k) {
    std::vector<std::pair<float, uint32_t>> by_distance;
    for (size_t j = 0; j < k_count; ++j)
      if (j != k) by_distance.push_back({sq_dist(centres[k], centres[j]), uint32_t(j)});
    const size_t three = std::min<size_t>(3, by_distance.size());
    const size_t six = std::min<size_t>(6, by_distance.size());
    std::partial_sort(by_distance.begin(), by_distance.begin() + six, by_distance.end());
    double ms = 0.0;
    for (size_t j = 0; j < three; ++j) ms += by_distance[j].first;
    float r = three > 0 ? float(std::sqrt(ms / double(three))) : 0.0f;
    if (!(r > 1e-4f)) r = fallback;
    nodes_[k] = {centres[k], r};
    radii[k] = r;
    for (size_t j = 0; j < six; ++j) links_[k].push_back(by_distance[j].second);
  }
  for (size_t k = 0; k < k_count; ++k)  // both ways
    for (uint32_t j : std::vector<uint32_t>(links_[k]))
      if (std::find(links_[j].begin(), links_[j].end(), uint32_t(k)) == links_[j].end()) links_[j].push_back(uint32_t(k));
  std::nth_element(radii.begin(), radii.begin() + long(k_count / 2), radii.end());
  spacing_ = radii[k_count / 2];
  views_.assign(frames, View{RigPose(k_count), std::vector<std::array<VectorAdam, 2>>(k_count), 0u});
}

RigPose NodeRig::estimate(size_t f, const CaptureOrder& order) const {
  if (learned(f)) return pose(f);
  RigPose out(nodes_.size());
  const CaptureOrder::Span s = order.around(f, [&](size_t i) { return learned(i); });
  if (s.none()) return out;
  const RigPose& a = pose(s.lo != CaptureOrder::kNone ? s.lo : s.hi);
  const RigPose& b = pose(s.hi != CaptureOrder::kNone ? s.hi : s.lo);
  for (size_t k = 0; k < out.size(); ++k)
    for (int c = 0; c < 3; ++c) {
      out[k].turn[c] = a[k].turn[c] + (b[k].turn[c] - a[k].turn[c]) * s.t;
      out[k].shift[c] = a[k].shift[c] + (b[k].shift[c] - a[k].shift[c]) * s.t;
    }
  return out;
}

void NodeRig::begin(size_t f, const CaptureOrder& order) {
  if (!learned(f)) views_.at(f).pose = estimate(f, order);
}

void NodeRig::set(size_t f, size_t node, const Vec3& turn, const Vec3& shift) {
  View& v = views_.at(f);
  v.pose.at(node) = {turn, shift};
  v.updates = std::max(v.updates, 1u);
}

void NodeRig::add_energy_gradient(size_t f, const RigEnergy& energy, const CaptureOrder& order,
                                  std::vector<double>& grad) const {
  // Each term is w * |r|^2 for a residual r linear (or, for a turn, linearised) in the
  // view's node motions; its gradient is 2 w J^T r. Shift residuals are divided by the
  // spacing s, so their weights carry 1 / s^2.
  const size_t K = nodes_.size();
  const RigPose& p = pose(f);
  const double inv_s2 = 1.0 / (double(spacing_) * double(spacing_));
  auto add = [&](size_t k, int part, const Vec3& r, double w) {
    for (int c = 0; c < 3; ++c) grad[k * 6 + part * 3 + c] += 2.0 * w * r[c];
  };
  for (size_t k = 0; k < K; ++k) {  // small
    add(k, 0, p[k].shift, energy.decay * inv_s2);
    add(k, 1, p[k].turn, energy.decay);
  }
  if (energy.rigidity > 0.0) {
    // Link k -> j: r = (n_j + s_j) - (n_k + s_k) - R_k (n_j - n_k). A turn u applied on top
    // of R_k moves R_k d by u x (R_k d), so dr = (R_k d) x u, J = [R_k d]x and
    // J^T r = -(R_k d) x r = r x (R_k d).
    for (size_t k = 0; k < K; ++k) {
      const Rotation Rk = Rotation::exp(p[k].turn);
      for (uint32_t j : links_[k]) {
        Vec3 d, r;
        for (int c = 0; c < 3; ++c) d[c] = double(nodes_[j].at[c]) - double(nodes_[k].at[c]);
        const Vec3 Rd = Rk.apply(d);
        for (int c = 0; c < 3; ++c) r[c] = d[c] + p[j].shift[c] - p[k].shift[c] - Rd[c];
        const double w = energy.rigidity * inv_s2;
        add(j, 0, r, w);
        add(k, 0, {-r[0], -r[1], -r[2]}, w);
        add(k, 1, cross(r, Rd), w);
      }
    }
  }
  if (energy.centring > 0.0) {
    // w views |mean|^2, the mean of the node's motion over the learned trained views and
    // this one: its gradient in this view's motion is 2 w mean = 2 (w / views) total.
    std::vector<NodeMotion> total(K);
    double views = 0.0;
    for (size_t g : order.trained()) {
      if (!learned(g) && g != f) continue;
      views += 1.0;
      for (size_t k = 0; k < K; ++k)
        for (int c = 0; c < 3; ++c) {
          total[k].shift[c] += pose(g)[k].shift[c];
          total[k].turn[c] += pose(g)[k].turn[c];
        }
    }
    const double share = 1.0 / std::max(views, 1.0);
    for (size_t k = 0; k < K; ++k) {
      add(k, 0, total[k].shift, energy.centring * inv_s2 * share);
      add(k, 1, total[k].turn, energy.centring * share);
    }
  }
  if (energy.smoothness > 0.0) {
    const CaptureOrder::Span s = order.around(f, [&](size_t i) { return learned(i); });
    for (size_t g : {s.lo, s.hi}) {
      if (g == CaptureOrder::kNone) continue;
      for (size_t k = 0; k < K; ++k) {
        Vec3 ds, dt;
        for (int c = 0; c < 3; ++c) {
          ds[c] = p[k].shift[c] - pose(g)[k].shift[c];
          dt[c] = p[k].turn[c] - pose(g)[k].turn[c];
        }
        add(k, 0, ds, energy.smoothness * inv_s2);
        add(k, 1, dt, energy.smoothness);
      }
    }
  }
}

double NodeRig::energy(size_t f, const RigEnergy& w, const CaptureOrder& order) const {
  const size_t K = nodes_.size();
  const RigPose& p = pose(f);
  const double inv_s2 = 1.0 / (double(spacing_) * double(spacing_));
  auto sq = [](const Vec3& v) { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; };
  double e = 0.0;
  for (size_t k = 0; k < K; ++k) e += w.decay * (sq(p[k].shift) * inv_s2 + sq(p[k].turn));
  for (size_t k = 0; k < K; ++k) {
    const Rotation Rk = Rotation::exp(p[k].turn);
    for (uint32_t j : links_[k]) {
      Vec3 d, r;
      for (int c = 0; c < 3; ++c) d[c] = double(nodes_[j].at[c]) - double(nodes_[k].at[c]);
      const Vec3 Rd = Rk.apply(d);
      for (int c = 0; c < 3; ++c) r[c] = d[c] + p[j].shift[c] - p[k].shift[c] - Rd[c];
      e += w.rigidity * inv_s2 * sq(r);
    }
  }
  if (w.centring > 0.0) {
    std::vector<NodeMotion> total(K);
    double views = 0.0;
    for (size_t g : order.trained()) {
      if (!learned(g) && g != f) continue;
      views += 1.0;
      for (size_t k = 0; k < K; ++k)
        for (int c = 0; c < 3; ++c) {
          total[k].shift[c] += pose(g)[k].shift[c];
          total[k].turn[c] += pose(g)[k].turn[c];
        }
    }
    // w |sum over views|^2 / views = w views |mean|^2: its gradient in one view's motion is
    // 2 w mean.
    const double share = 1.0 / std::max(views, 1.0);
    for (size_t k = 0; k < K; ++k) e += w.centring * share * (sq(total[k].shift) * inv_s2 + sq(total[k].turn));
  }
  if (w.smoothness > 0.0) {
    const CaptureOrder::Span s = order.around(f, [&](size_t i) { return learned(i); });
    for (size_t g : {s.lo, s.hi}) {
      if (g == CaptureOrder::kNone) continue;
      for (size_t k = 0; k < K; ++k) {
        Vec3 ds, dt;
        for (int c = 0; c < 3; ++c) {
          ds[c] = p[k].shift[c] - pose(g)[k].shift[c];
          dt[c] = p[k].turn[c] - pose(g)[k].turn[c];
        }
        e += w.smoothness * (sq(ds) * inv_s2 + sq(dt));
      }
    }
  }
  return e;
}

std::vector<double> NodeRig::energy_gradient(size_t f, const RigEnergy& w, const CaptureOrder& order) const {
  std::vector<double> grad(nodes_.size() * 6, 0.0);
  add_energy_gradient(f, w, order, grad);
  return grad;
}

void NodeRig::learn(size_t f, const double* image_grad, const RigEnergy& energy, double shift_rate, double turn_rate,
                    const CaptureOrder& order) {
  const size_t K = nodes_.size();
  std::vector<double> grad(image_grad, image_grad + K * 6);
  add_energy_gradient(f, energy, order, grad);
  View& v = views_.at(f);
  const uint32_t n = ++v.updates;
  constexpr double b1 = 0.9, b2 = 0.999;
  const double c1 = 1.0 / (1.0 - std::pow(b1, double(n)));
  const double c2 = 1.0 / (1.0 - std::pow(b2, double(n)));
  for (size_t k = 0; k < K; ++k)
    for (int part = 0; part < 2; ++part) {
      VectorAdam& a = v.adam[k][part];
      double mean_sq = 0.0;
      for (int c = 0; c < 3; ++c) {
        const double g = grad[k * 6 + part * 3 + c];
        a.m[c] += (1.0 - b1) * (g - a.m[c]);
        mean_sq += g * g / 3.0;
      }
      a.v += (1.0 - b2) * (mean_sq - a.v);
      if (!(a.v > 0.0)) continue;
      const double rate = part == 0 ? shift_rate : turn_rate;
      const double scale = rate * c1 / (std::sqrt(a.v * c2) + 1e-30);
      Vec3& value = part == 0 ? v.pose[k].shift : v.pose[k].turn;
      for (int c = 0; c < 3; ++c) value[c] -= scale * a.m[c];
    }
}

std::vector<float> NodeRig::table(const RigPose& pose) const {
  std::vector<float> out(nodes_.size() * 20, 0.0f);
  for (size_t k = 0; k < nodes_.size(); ++k) {
    double R[9];
    Rotation::exp(pose[k].turn).to_matrix(R);
    float* o = &out[k * 20];
    for (int r = 0; r < 3; ++r) {
      const double centre = double(nodes_[k].at[r]) + pose[k].shift[r];
      double b = centre;
      for (int c = 0; c < 3; ++c) {
        o[r * 4 + c] = float(R[r * 3 + c]);
        b -= R[r * 3 + c] * double(nodes_[k].at[c]);
      }
      o[r * 4 + 3] = float(b);
      o[12 + r] = float(pose[k].turn[r]);
      o[16 + r] = float(centre);
    }
  }
  return out;
}

NodeRig::Spread NodeRig::spread(const std::vector<size_t>& frames) const {
  Spread out;
  size_t n = 0;
  for (size_t f : frames) {
    if (!learned(f)) continue;
    out.updates += updates(f);
    for (const NodeMotion& m : pose(f)) {
      const double s = length(m.shift), t = length(m.turn) * 180.0 / kPi;
      out.shift_mean += s;
      out.turn_mean += t;
      out.shift_max = std::max(out.shift_max, s);
      out.turn_max = std::max(out.turn_max, t);
      ++n;
    }
  }
  if (n > 0) {
    out.shift_mean /= double(n);
    out.turn_mean /= double(n);
  }
  return out;
}

}  // namespace gs::refine
