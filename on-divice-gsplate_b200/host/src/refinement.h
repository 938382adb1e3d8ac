// Per-view corrections gs::Trainer learns beside the gaussians: a rigid camera correction
// and three exposure gains per dataset frame, plus the capture-order lookups that fill in
// frames that were never trained on. The GPU step supplies the gradients and fit sums
// (gs_step_result.pose_grad / .fit); everything here is small host-side state.
//
// Conventions. A correction (turn U, shift s) acts in camera axes after the dataset's
// world -> camera transform: x_cam = U (R x + t) + s, i.e. the camera becomes [U R | U t + s].
// A step with rotation vector w and translation d is applied on the left:
// (U, s) <- (exp([w]x) U, exp([w]x) s + d); the GPU's pose gradient is dL/d(d, w) at d = w = 0.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <vector>

#include "gs/camera.h"

namespace gs::refine {

using Vec3 = std::array<double, 3>;

// A rotation as a unit quaternion (w, x, y, z).
struct Rotation {
  std::array<double, 4> q{1.0, 0.0, 0.0, 0.0};

  static Rotation exp(const Vec3& v);  // the rotation by |v| radians about v
  Vec3 log() const;                    // its rotation vector, angle in [0, pi]
  Rotation after(const Rotation& first) const;  // `first`, then this
  Vec3 apply(const Vec3& v) const;
  void to_matrix(double m[9]) const;  // row-major
  double degrees() const;
  // Spherical interpolation on the shorter arc (t = 0: a, t = 1: b).
  static Rotation slerp(const Rotation& a, const Rotation& b, double t);
};

struct RigidFix {
  Rotation turn;
  Vec3 shift{0.0, 0.0, 0.0};

  // This correction followed by the step (d, w): (exp(w) U, exp(w) s + d).
  RigidFix then(const Vec3& d, const Vec3& w) const;
  // A camera with this correction applied (position recomputed as -R^T t).
  Camera apply(const Camera& camera) const;
  static RigidFix blend(const RigidFix& a, const RigidFix& b, double t);
};

// Adam over a fixed-size vector, its bias correction counted by its own updates.
// beta1 = 0.9, beta2 = 0.999 (the step's own constants, trainer.cpp:68-69).
template <size_t N>
struct Adam {
  std::array<double, N> m{}, v{};
  uint32_t updates = 0;
  // Records `grad` and returns the step -rate_i mhat_i / (sqrt(vhat_i) + tiny), 0 where
  // no gradient has been seen.
  std::array<double, N> step(const std::array<double, N>& grad, const std::array<double, N>& rate);
};

// Trained frames around each frame of a capture, in capture order.
class CaptureOrder {
 public:
  static constexpr size_t kNone = ~size_t(0);
  void build(size_t frames, const std::vector<size_t>& trained);
  // The nearest trained frames lo < f < hi for which `usable` holds (kNone when there is
  // none on that side) and the weight of hi, (f - lo) / (hi - lo): 0 or 1 when only one
  // side has one. f itself is never returned.
  struct Span {
    size_t lo = kNone, hi = kNone;
    double t = 0.0;
    bool none() const { return lo == kNone && hi == kNone; }
  };
  Span around(size_t f, const std::function<bool(size_t)>& usable) const;
  const std::vector<size_t>& trained() const { return trained_; }

 private:
  std::vector<size_t> trained_;  // ascending
  size_t frames_ = 0;
};

// Camera corrections of every frame.
class PoseTable {
 public:
  void reset(size_t frames) { rows_.assign(frames, Row{}); }
  bool learned(size_t f) const { return rows_.at(f).learned; }
  const RigidFix& fix(size_t f) const { return rows_.at(f).fix; }
  // Sets a frame's correction (an alignment result); it then counts as learned.
  void assign(size_t f, const RigidFix& fix);
  // One Adam step on frame f's correction from its pose gradient (dL/dd xyz, dL/dw xyz);
  // rates: shift per update (dataset units), turn per update (radians).
  void learn(size_t f, const double grad[6], double shift_rate, double turn_rate);
  // Frame f's own correction once learned, else the blend of the nearest learned frames
  // around it in capture order, else none.
  RigidFix estimate(size_t f, const CaptureOrder& order) const;
  struct Spread {
    double shift_mean = 0.0, shift_max = 0.0;  // camera centre moved, dataset units
    double turn_mean = 0.0, turn_max = 0.0;    // degrees
    uint32_t updates = 0;
  };
  // Over `frames`, the learned ones; base(f) is a frame's camera without correction.
  Spread spread(const std::vector<size_t>& frames, const std::function<Camera(size_t)>& base) const;

 private:
  struct Row {
    RigidFix fix;
    Adam<6> adam;  // shift xyz, turn xyz
    bool learned = false;
  };
  std::vector<Row> rows_;
};

// A view's photometric alignment: minimise its loss over the correction by steps along
// the normalised pose gradient, turns weighted by `reach` (a turn of w moves the image
// about as a shift of reach * w). `probe` renders a correction and returns false if it
// could not; it fills the loss and the pose gradient there. Starts at each of `starts`
// (one evaluation each), then spends the rest of `budget` on steps from the best point
// seen: a step that lowers the loss is taken and the next one is twice as long, one that
// does not is dropped and the length quartered. Never returns a correction worse than the
// best start.
RigidFix align(const std::function<bool(const RigidFix&, double& loss, double grad[6])>& probe,
               const std::vector<RigidFix>& starts, uint32_t budget, double first_step, double reach);

// Exposure gains of every frame: the photo is divided by them before the loss.
class GainTable {
 public:
  void reset(size_t frames) { rows_.assign(frames, Row{}); }
  // A trained view's fit sums from the forward pass (gs_step_result.fit: sum render^2 per
  // channel, opaque pixels, sum render * photo per channel): the gain that maps the render
  // onto the photo, sum(render * photo) / sum(render^2), clamped to [1/4, 4], enters the
  // frame's log gain at `rate` (the first measurement as is). Views with fewer than 500
  // opaque pixels are not measured.
  void observe(size_t f, const double fit[8], double rate);
  bool measured(size_t f) const { return rows_.at(f).count > 0; }
  // Only ratios between views are fixed by photos, so the gains used are centred: divided by
  // their geometric mean over the measured trained views. A frame not measured takes the
  // blend of the measured ones around it in capture order; 1 when nothing is measured.
  std::array<float, 3> gains(size_t f, const CaptureOrder& order) const;
  struct Spread {
    double low = 1.0, high = 1.0;  // 5th and 95th percentile luminance gain
    double tint = 0.0;             // standard deviation of (red + blue) / 2 / green
    uint32_t updates = 0;
  };
  Spread spread(const CaptureOrder& order) const;

 private:
  struct Row {
    Vec3 log{0.0, 0.0, 0.0};
    uint32_t count = 0;
  };
  Vec3 centre(const CaptureOrder& order) const;
  std::vector<Row> rows_;
};

}  // namespace gs::refine
