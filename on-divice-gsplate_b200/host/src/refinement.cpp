// Camera corrections and exposure gains (refinement.h): quaternion rigid corrections with
// Adam, the alignment search, and centred per-channel gains.
#include "refinement.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace gs::refine {

namespace {

constexpr double kPi = 3.14159265358979323846;

double norm3(const Vec3& v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

}  // namespace

// ---- rotations and rigid corrections ----

Rotation Rotation::exp(const Vec3& v) {
  const double angle = norm3(v);
  Rotation r;
  if (angle < 1e-12) {
    // First order: (1, v / 2), normalised.
    const double n = std::sqrt(1.0 + 0.25 * angle * angle);
    r.q = {1.0 / n, 0.5 * v[0] / n, 0.5 * v[1] / n, 0.5 * v[2] / n};
    return r;
  }
  const double s = std::sin(0.5 * angle) / angle;
  r.q = {std::cos(0.5 * angle), s * v[0], s * v[1], s * v[2]};
  return r;
}

Vec3 Rotation::log() const {
  // q and -q are the same rotation: take w >= 0 for the angle in [0, pi].
  const double sign = q[0] < 0.0 ? -1.0 : 1.0;
  const Vec3 u{sign * q[1], sign * q[2], sign * q[3]};
  const double s = norm3(u);
  if (s < 1e-12) return {2.0 * u[0], 2.0 * u[1], 2.0 * u[2]};
  const double angle = 2.0 * std::atan2(s, sign * q[0]);
  return {angle * u[0] / s, angle * u[1] / s, angle * u[2] / s};
}

Rotation Rotation::after(const Rotation& first) const {
  const auto& a = q;
  const auto& b = first.q;
  Rotation r;
  r.q = {a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3], a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
         a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1], a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0]};
  const double n = std::sqrt(r.q[0] * r.q[0] + r.q[1] * r.q[1] + r.q[2] * r.q[2] + r.q[3] * r.q[3]);
  for (double& c : r.q) c /= n;
  return r;
}

void Rotation::to_matrix(double m[9]) const {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  m[0] = 1.0 - 2.0 * (y * y + z * z);
  m[1] = 2.0 * (x * y - w * z);
  m[2] = 2.0 * (x * z + w * y);
  m[3] = 2.0 * (x * y + w * z);
  m[4] = 1.0 - 2.0 * (x * x + z * z);
  m[5] = 2.0 * (y * z - w * x);
  m[6] = 2.0 * (x * z - w * y);
  m[7] = 2.0 * (y * z + w * x);
  m[8] = 1.0 - 2.0 * (x * x + y * y);
}

Vec3 Rotation::apply(const Vec3& v) const {
  double m[9];
  to_matrix(m);
  return {m[0] * v[0] + m[1] * v[1] + m[2] * v[2], m[3] * v[0] + m[4] * v[1] + m[5] * v[2],
          m[6] * v[0] + m[7] * v[1] + m[8] * v[2]};
}

double Rotation::degrees() const { return norm3(log()) * 180.0 / kPi; }

Rotation Rotation::slerp(const Rotation& a, const Rotation& b, double t) {
  double dot = a.q[0] * b.q[0] + a.q[1] * b.q[1] + a.q[2] * b.q[2] + a.q[3] * b.q[3];
  std::array<double, 4> end = b.q;
  if (dot < 0.0) {  // the shorter arc
    dot = -dot;
    for (double& c : end) c = -c;
  }
  double wa = 1.0 - t, wb = t;
  if (dot < 1.0 - 1e-9) {
    const double theta = std::acos(std::min(dot, 1.0));
    wa = std::sin((1.0 - t) * theta) / std::sin(theta);
    wb = std::sin(t * theta) / std::sin(theta);
  }
  Rotation r;
  double n = 0.0;
  for (int k = 0; k < 4; ++k) {
    r.q[k] = wa * a.q[k] + wb * end[k];
    n += r.q[k] * r.q[k];
  }
  n = std::sqrt(n);
  for (double& c : r.q) c /= n;
  return r;
}

RigidFix RigidFix::then(const Vec3& d, const Vec3& w) const {
  const Rotation step = Rotation::exp(w);
  RigidFix out;
  out.turn = step.after(turn);
  const Vec3 moved = step.apply(shift);
  for (int c = 0; c < 3; ++c) out.shift[c] = moved[c] + d[c];
  return out;
}

Camera RigidFix::apply(const Camera& camera) const {
  double U[9];
  turn.to_matrix(U);
  Camera out = camera;
  for (int r = 0; r < 3; ++r) {
    double t = shift[r];
    for (int c = 0; c < 3; ++c) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += U[r * 3 + k] * double(camera.rotation[k * 3 + c]);
      out.rotation[r * 3 + c] = float(v);
      t += U[r * 3 + c] * double(camera.translation[c]);
    }
    out.translation[r] = float(t);
  }
  for (int c = 0; c < 3; ++c) {
    double p = 0.0;
    for (int r = 0; r < 3; ++r) p -= double(out.rotation[r * 3 + c]) * double(out.translation[r]);
    out.position[c] = float(p);
  }
  return out;
}

RigidFix RigidFix::blend(const RigidFix& a, const RigidFix& b, double t) {
  RigidFix out;
  out.turn = Rotation::slerp(a.turn, b.turn, t);
  for (int c = 0; c < 3; ++c) out.shift[c] = a.shift[c] + (b.shift[c] - a.shift[c]) * t;
  return out;
}

template <size_t N>
std::array<double, N> Adam<N>::step(const std::array<double, N>& grad, const std::array<double, N>& rate) {
  constexpr double b1 = 0.9, b2 = 0.999;
  ++updates;
  const double c1 = 1.0 / (1.0 - std::pow(b1, double(updates)));
  const double c2 = 1.0 / (1.0 - std::pow(b2, double(updates)));
  std::array<double, N> out{};
  for (size_t i = 0; i < N; ++i) {
    m[i] += (1.0 - b1) * (grad[i] - m[i]);
    v[i] += (1.0 - b2) * (grad[i] * grad[i] - v[i]);
    out[i] = v[i] > 0.0 ? -rate[i] * (m[i] * c1) / (std::sqrt(v[i] * c2) + 1e-30) : 0.0;
  }
  return out;
}

template struct Adam<6>;

// ---- capture order ----

void CaptureOrder::build(size_t frames, const std::vector<size_t>& trained) {
  frames_ = frames;
  trained_ = trained;
  std::sort(trained_.begin(), trained_.end());
}

CaptureOrder::Span CaptureOrder::around(size_t f, const std::function<bool(size_t)>& usable) const {
  Span s;
  auto it = std::lower_bound(trained_.begin(), trained_.end(), f);
  for (auto up = it; up != trained_.end(); ++up)
    if (*up != f && usable(*up)) {
      s.hi = *up;
      break;
    }
  for (auto down = it; down != trained_.begin();) {
    --down;
    if (usable(*down)) {
      s.lo = *down;
      break;
    }
  }
  if (s.lo != kNone && s.hi != kNone) s.t = double(f - s.lo) / double(s.hi - s.lo);
  else s.t = s.hi != kNone ? 1.0 : 0.0;
  return s;
}

// ---- camera corrections ----

void PoseTable::assign(size_t f, const RigidFix& fix) {
  Row& row = rows_.at(f);
  row.fix = fix;
  row.learned = true;
}

void PoseTable::learn(size_t f, const double grad[6], double shift_rate, double turn_rate) {
  Row& row = rows_.at(f);
  std::array<double, 6> g{}, rate{};
  for (int i = 0; i < 6; ++i) {
    g[i] = grad[i];
    rate[i] = i < 3 ? shift_rate : turn_rate;
  }
  const std::array<double, 6> step = row.adam.step(g, rate);
  row.fix = row.fix.then({step[0], step[1], step[2]}, {step[3], step[4], step[5]});
  row.learned = true;
}

RigidFix PoseTable::estimate(size_t f, const CaptureOrder& order) const {
  if (learned(f)) return fix(f);
  const CaptureOrder::Span s = order.around(f, [&](size_t i) { return learned(i); });
  if (s.none()) return RigidFix{};
  if (s.lo == CaptureOrder::kNone) return fix(s.hi);
  if (s.hi == CaptureOrder::kNone) return fix(s.lo);
  return RigidFix::blend(fix(s.lo), fix(s.hi), s.t);
}

PoseTable::Spread PoseTable::spread(const std::vector<size_t>& frames,
                                    const std::function<Camera(size_t)>& base) const {
  Spread out;
  uint32_t n = 0;
  for (size_t f : frames) {
    const Row& row = rows_.at(f);
    if (!row.learned) continue;
    const Camera a = base(f), b = row.fix.apply(a);
    double moved = 0.0;
    for (int c = 0; c < 3; ++c) moved += (double(b.position[c]) - a.position[c]) * (double(b.position[c]) - a.position[c]);
    moved = std::sqrt(moved);
    const double turned = row.fix.turn.degrees();
    out.shift_mean += moved;
    out.turn_mean += turned;
    out.shift_max = std::max(out.shift_max, moved);
    out.turn_max = std::max(out.turn_max, turned);
    out.updates += row.adam.updates;
    ++n;
  }
  if (n > 0) {
    out.shift_mean /= n;
    out.turn_mean /= n;
  }
  return out;
}

RigidFix align(const std::function<bool(const RigidFix&, double& loss, double grad[6])>& probe,
               const std::vector<RigidFix>& starts, uint32_t budget, double first_step, double reach) {
  RigidFix best;
  double best_loss = std::numeric_limits<double>::infinity(), best_grad[6] = {0, 0, 0, 0, 0, 0};
  uint32_t used = 0;
  auto consider = [&](const RigidFix& fix) {
    ++used;
    double loss = 0.0, grad[6];
    if (!probe(fix, loss, grad) || !(loss < best_loss)) return false;
    best = fix;
    best_loss = loss;
    std::copy(grad, grad + 6, best_grad);
    return true;
  };
  for (const RigidFix& s : starts) {
    if (used >= budget) break;
    consider(s);
  }
  if (!(best_loss < std::numeric_limits<double>::infinity())) return RigidFix{};
  double length = first_step;
  while (used < budget) {
    // The gradient in (shift, reach * turn) units, so both parts move the image alike.
    const double g[6] = {best_grad[0], best_grad[1], best_grad[2], best_grad[3] / reach, best_grad[4] / reach,
                         best_grad[5] / reach};
    double norm = 0.0;
    for (double v : g) norm += v * v;
    if (!(norm > 0.0)) break;
    norm = std::sqrt(norm);
    const Vec3 d{-length * g[0] / norm, -length * g[1] / norm, -length * g[2] / norm};
    const Vec3 w{-length * g[3] / norm / reach, -length * g[4] / norm / reach, -length * g[5] / norm / reach};
    length *= consider(best.then(d, w)) ? 2.0 : 0.25;
  }
  return best;
}

// ---- exposure gains ----

void GainTable::observe(size_t f, const double fit[8], double rate) {
  if (fit[3] < 500.0) return;
  Row& row = rows_.at(f);
  const double r = row.count == 0 ? 1.0 : std::clamp(rate, 0.0, 1.0);
  for (int c = 0; c < 3; ++c) {
    if (!(fit[c] > 1e-9)) continue;
    const double measured = std::log(std::clamp(fit[4 + c] / fit[c], 0.25, 4.0));
    row.log[c] += r * (measured - row.log[c]);
  }
  ++row.count;
}

Vec3 GainTable::centre(const CaptureOrder& order) const {
  Vec3 sum{0.0, 0.0, 0.0};
  size_t n = 0;
  for (size_t f : order.trained()) {
    if (!measured(f)) continue;
    for (int c = 0; c < 3; ++c) sum[c] += rows_[f].log[c];
    ++n;
  }
  if (n > 0)
    for (double& v : sum) v /= double(n);
  return sum;
}

std::array<float, 3> GainTable::gains(size_t f, const CaptureOrder& order) const {
  std::array<float, 3> out{1.0f, 1.0f, 1.0f};
  if (f >= rows_.size()) return out;
  const bool any = std::any_of(order.trained().begin(), order.trained().end(), [&](size_t i) { return measured(i); });
  if (!any) return out;
  const Vec3 mid = centre(order);
  Vec3 log = rows_[f].log;
  if (!measured(f)) {
    const CaptureOrder::Span s = order.around(f, [&](size_t i) { return measured(i); });
    if (s.none()) return out;
    const Vec3& a = rows_[s.lo != CaptureOrder::kNone ? s.lo : s.hi].log;
    const Vec3& b = rows_[s.hi != CaptureOrder::kNone ? s.hi : s.lo].log;
    for (int c = 0; c < 3; ++c) log[c] = a[c] + (b[c] - a[c]) * s.t;
  }
  for (int c = 0; c < 3; ++c) out[c] = float(std::exp(log[c] - mid[c]));
  return out;
}

GainTable::Spread GainTable::spread(const CaptureOrder& order) const {
  Spread out;
  std::vector<double> luma, tint;
  for (size_t f : order.trained()) {
    if (!measured(f)) continue;
    out.updates += rows_[f].count;
    const std::array<float, 3> g = gains(f, order);
    luma.push_back(0.299 * g[0] + 0.587 * g[1] + 0.114 * g[2]);  // Rec. 601 luma weights
    tint.push_back(0.5 * (double(g[0]) + g[2]) / std::max(double(g[1]), 1e-6));
  }
  if (luma.empty()) return out;
  std::sort(luma.begin(), luma.end());
  auto quantile = [&](double p) {  // linear between the order statistics
    const double x = p * double(luma.size() - 1);
    const size_t i = size_t(x);
    const double frac = x - double(i);
    return i + 1 < luma.size() ? luma[i] + (luma[i + 1] - luma[i]) * frac : luma[i];
  };
  out.low = quantile(0.05);
  out.high = quantile(0.95);
  if (tint.size() > 1) {
    double mean = 0.0, sq = 0.0;
    for (double x : tint) mean += x;
    mean /= double(tint.size());
    for (double x : tint) sq += (x - mean) * (x - mean);
    out.tint = std::sqrt(sq / double(tint.size() - 1));
  }
  return out;
}

}  // namespace gs::refine
