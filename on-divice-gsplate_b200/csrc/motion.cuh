// Subject motion on the device (train_motion.glsl): the model is the subject at rest; in a
// view each control node k moves rigidly, x -> R_k x + b_k with b_k = c_k - R_k n_k (a turn
// about the node's rest position n_k, then a shift to c_k), and a slot follows its 4 nearest
// nodes blended by weight:
//   position     x = sum_k w_k (R_k p + b_k),        dx/dp = A = sum_k w_k R_k
//   orientation  turned by U = exp([sum_k w_k turn_k]x)
#pragma once

#include "gs_common.cuh"

namespace gsk {

constexpr uint32_t kMaxMotionNodes = GS_MAX_MOTION_NODES;

// One node's motion in one view: the rows of [R | b], the turn vector, where it moved to.
struct MotionNode {
  float4 row[3];
  float4 turn;
  float4 moved;
};
static_assert(sizeof(MotionNode) == 80, "20 floats per node, as gs_set_view_motion takes them");

struct Motion {
  uint32_t nodes = 0;                 // 0: no motion anywhere
  const float4* rest = nullptr;       // per node: rest position xyz, 1 / (2 r^2)
  uint4* bind = nullptr;              // 2 per slot: node indices, weights (float bits)
  const MotionNode* views = nullptr;  // kMaxMotionNodes per view of the step
};

// U = exp([w]x) = I + a [w]x + b (w w^T - |w|^2 I), a = sin t / t, b = (1 - cos t) / t^2
// (series below t = 1e-4, as train_motion.glsl:13-20).
__device__ __forceinline__ void turn_matrix(float wx, float wy, float wz, float U[3][3]) {
  const float t2 = wx * wx + wy * wy + wz * wz, t = sqrtf(t2);
  const float a = t > 1e-4f ? sinf(t) / t : 1.0f - t2 / 6.0f;
  const float b = t > 1e-4f ? (1.0f - cosf(t)) / t2 : 0.5f - t2 / 24.0f;
  const float w[3] = {wx, wy, wz};
  const float K[3][3] = {{0.0f, -wz, wy}, {wz, 0.0f, -wx}, {-wy, wx, 0.0f}};
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) U[r][c] = (r == c ? 1.0f - b * t2 : 0.0f) + a * K[r][c] + b * w[r] * w[c];
}

// Where slot i (rest position p) is in a view: x, the orientation's turn U and A = dx/dp
// (train_motion.glsl:33-49).
struct Deformed {
  float x[3];
  float U[3][3];
  float A[3][3];
};

__device__ __forceinline__ void deform(const Motion& m, const MotionNode* view, uint32_t i, float px, float py,
                                       float pz, Deformed& d) {
  const uint4 nodes = m.bind[2u * i];
  const uint4 wb = m.bind[2u * i + 1u];
  const uint32_t nk[4] = {nodes.x, nodes.y, nodes.z, nodes.w};
  const float wk[4] = {__uint_as_float(wb.x), __uint_as_float(wb.y), __uint_as_float(wb.z), __uint_as_float(wb.w)};
  float turn[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    d.x[r] = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c) d.A[r][c] = 0.0f;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (wk[j] == 0.0f) continue;
    const MotionNode& n = view[nk[j]];
    const float4 rows[3] = {n.row[0], n.row[1], n.row[2]};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      d.x[r] += wk[j] * (rows[r].x * px + rows[r].y * py + rows[r].z * pz + rows[r].w);
      d.A[r][0] += wk[j] * rows[r].x;
      d.A[r][1] += wk[j] * rows[r].y;
      d.A[r][2] += wk[j] * rows[r].z;
    }
    turn[0] += wk[j] * n.turn.x;
    turn[1] += wk[j] * n.turn.y;
    turn[2] += wk[j] * n.turn.z;
  }
  turn_matrix(turn[0], turn[1], turn[2], d.U);
}

// No motion: x = p, U = A = I.
__device__ __forceinline__ void at_rest(float px, float py, float pz, Deformed& d) {
  d.x[0] = px;
  d.x[1] = py;
  d.x[2] = pz;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) d.U[r][c] = d.A[r][c] = r == c ? 1.0f : 0.0f;
}

}  // namespace gsk
