// Subject motion for gs::Trainer: a rig of control nodes spread over the subject, each
// moved per view by a rigid motion (a turn about the node and a shift). The GPU blends the
// four nearest nodes' motions into every gaussian (gs_motion_bind, gs_set_view_motion) and
// sums the image loss's gradient per node (GS_FLAG_MOTION_GRAD, gs_motion_gradient); this
// file keeps the nodes, each view's motions and their optimiser, and the regularising
// energies that keep motions small, locally rigid, smooth across neighbouring views and
// centred on the rest pose.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "refinement.h"

namespace gs::refine {

struct NodeMotion {
  Vec3 turn{0.0, 0.0, 0.0};   // rotation vector about the node, radians
  Vec3 shift{0.0, 0.0, 0.0};  // translation of the node, dataset units
};
using RigPose = std::vector<NodeMotion>;  // one per node

// Weights of the regularising energies, each in units where a shift of one node spacing
// counts like a turn of one radian.
struct RigEnergy {
  double decay = 0.0;       // sum over nodes of |shift|^2 / s^2 + |turn|^2
  double rigidity = 0.0;    // sum over linked nodes of |where k's motion takes j - where j went|^2 / s^2
  double smoothness = 0.0;  // difference to the learned views before and after in capture order
  double centring = 0.0;    // the mean motion over the learned views, pulled to zero
};

class NodeRig {
 public:
  struct Node {
    std::array<float, 3> at;
    float radius;  // gaussians weigh a node by exp(-d^2 / (2 radius^2))
  };

  // Up to `count` nodes over `xyz` (three floats per point; at most 20000 points are used,
  // evenly strided): farthest-point seeds from the point nearest the centroid, refined by
  // Lloyd iterations until no point changes node (at most 25). A node's radius is the root
  // mean square distance to its three nearest nodes (`fallback` when that is degenerate);
  // each node is linked to its six nearest, and links go both ways. Views start at rest.
  void place(const std::vector<float>& xyz, size_t count, size_t frames, float fallback);
  bool empty() const { return nodes_.empty(); }
  size_t size() const { return nodes_.size(); }
  const std::vector<Node>& nodes() const { return nodes_; }
  float spacing() const { return spacing_; }  // the median radius

  bool learned(size_t f) const { return views_.at(f).updates > 0; }
  uint32_t updates(size_t f) const { return views_.at(f).updates; }
  const RigPose& pose(size_t f) const { return views_.at(f).pose; }
  // A view's motions once learned, else the blend of the nearest learned views around it in
  // capture order, else rest.
  RigPose estimate(size_t f, const CaptureOrder& order) const;
  // Before a view's first update: it starts from that estimate.
  void begin(size_t f, const CaptureOrder& order);
  // Sets one node's motion in a view, which then counts as learned.
  void set(size_t f, size_t node, const Vec3& turn, const Vec3& shift);
  // One update of view f: the image loss's gradient (6 per node: dL/dshift xyz, dL/dturn
  // xyz) plus the energies' gradients, then an Adam step whose second moment is shared by
  // the three components of each node's shift and of its turn (the step keeps the
  // vector's direction). Rates per update: shift in dataset units, turn in radians.
  void learn(size_t f, const double* image_grad, const RigEnergy& energy, double shift_rate, double turn_rate,
             const CaptureOrder& order);
  // The regularising energy of view f's motions and its gradient (6 per node: shift xyz,
  // turn xyz, the turn's as a rotation applied on top of the node's).
  double energy(size_t f, const RigEnergy& weights, const CaptureOrder& order) const;
  std::vector<double> energy_gradient(size_t f, const RigEnergy& weights, const CaptureOrder& order) const;
  // The GPU's node table of a pose (gs_set_view_motion): per node [R | b] (12 floats),
  // turn (4), moved centre (4), with R = exp(turn), c = node + shift, b = c - R node.
  std::vector<float> table(const RigPose& pose) const;

  struct Spread {
    double shift_mean = 0.0, shift_max = 0.0;  // dataset units
    double turn_mean = 0.0, turn_max = 0.0;    // degrees
    uint32_t updates = 0;
  };
  Spread spread(const std::vector<size_t>& frames) const;

 private:
  struct VectorAdam {  // first moment per component, one second moment per 3-vector
    Vec3 m{0.0, 0.0, 0.0};
    double v = 0.0;
  };
  struct View {
    RigPose pose;
    std::vector<std::array<VectorAdam, 2>> adam;  // per node: shift, turn
    uint32_t updates = 0;
  };
  // Adds the energies' gradients of view f to grad (6 per node).
  void add_energy_gradient(size_t f, const RigEnergy& energy, const CaptureOrder& order,
                           std::vector<double>& grad) const;

  std::vector<Node> nodes_;
  std::vector<std::vector<uint32_t>> links_;
  float spacing_ = 1.0f;
  std::vector<View> views_;
};

}  // namespace gs::refine
