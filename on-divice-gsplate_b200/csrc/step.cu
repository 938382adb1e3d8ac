// Optimizer side of the step: per-gaussian pair sums (train_pair_sum.comp:17-32), the
// projection backward fused with Adam on all parameters (train_step.glsl:62-240 and
// train_step_sh.comp:21-44), adaptive density control (train_densify_mark.comp,
// train_densify_spawn.comp) and the opacity reset (train_reset_opacity.comp).
//
// The step back-propagates every view's summed 2D gradient through that view's projection
// (views of one step add up) and takes one Adam step on the active SH coefficients
// (k_step_sh, first: it also produces the position gradient through the SH view
// direction) and on the 16 parameters (k_step_geometry). HBM-bound: parameters, SH and
// both moment sets are read and written once per step.
#include <algorithm>
#include <utility>

#include "gs_kernels.h"

namespace gsk {
namespace {

struct PairSumArgs {
  uint32_t n_items;
  const uint32_t* order;   // items (view * cap + slot) in depth order
  const uint32_t* first;   // their first pair, in the same order
  const float4* pair_grads;
  float4* grad2d;
  const uint32_t* d_pairs;
  uint32_t accept;
};

// Items in depth order, so the 32 items of a warp own one contiguous run of pairs (the
// emit order); an item's count is the gap to the next item's first pair. The warp streams
// that run through shared memory kSumChunk pairs at a time, with coalesced loads and the
// next chunk's loads in flight while the lanes add the current one; each lane adds its own
// item's pairs one after another from zero, the order of train_pair_sum.comp:24-29. Items
// that drew no pair are skipped: the step reads grad2d only where tiles > 0.
constexpr uint32_t kSumChunk = 64;
constexpr uint32_t kSumLoads = kSumChunk * 3u / 32u;  // float4 per lane per chunk
constexpr uint32_t kSumWarps = 8;

__global__ void __launch_bounds__(kSumWarps * 32) k_pair_sum(PairSumArgs a) {
  __shared__ float4 s_chunk[kSumWarps][kSumChunk * 3u];
  const uint32_t total = *a.d_pairs;
  if (total > a.accept) return;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t base = (blockIdx.x * kSumWarps + warp) * 32u;
  if (base >= a.n_items) return;
  const uint32_t idx = base + lane;
  // Lanes past the last item own the empty run [total, total).
  const uint32_t first = idx < a.n_items ? a.first[idx] : total;
  uint32_t end = __shfl_down_sync(0xffffffffu, first, 1);
  if (lane == 31u) end = base + 32u < a.n_items ? a.first[base + 32u] : total;
  const uint32_t r0 = __shfl_sync(0xffffffffu, first, 0), r1 = __shfl_sync(0xffffffffu, end, 31);
  if (r0 == r1) return;
  float4* buf = s_chunk[warp];
  const float4* src = a.pair_grads;
  float4 v[kSumLoads];
  auto load = [&](uint32_t c0) {
    const uint32_t n = min(kSumChunk, r1 - c0) * 3u;
    const float4* p = src + size_t(c0) * 3u;
#pragma unroll
    for (uint32_t j = 0; j < kSumLoads; ++j) {
      const uint32_t k = lane + 32u * j;
      v[j] = k < n ? p[k] : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f), s1 = s0, s2 = s0;
  load(r0);
  for (uint32_t c0 = r0; c0 < r1; c0 += kSumChunk) {
    __syncwarp();
#pragma unroll
    for (uint32_t j = 0; j < kSumLoads; ++j) buf[lane + 32u * j] = v[j];
    __syncwarp();
    if (r1 - c0 > kSumChunk) load(c0 + kSumChunk);
    const uint32_t lo = max(first, c0), hi = min(end, c0 + kSumChunk);
    for (uint32_t q = lo; q < hi; ++q) {
      const float4* t = buf + (q - c0) * 3u;
      const float4 x = t[0], y = t[1], z = t[2];
      s0.x += x.x; s0.y += x.y; s0.z += x.z; s0.w += x.w;
      s1.x += y.x; s1.y += y.y; s1.z += y.z; s1.w += y.w;
      s2.x += z.x; s2.y += z.y; s2.z += z.z; s2.w += z.w;
    }
  }
  if (end == first) return;
  const size_t g = a.order[idx];
  a.grad2d[g * 3u] = s0;
  a.grad2d[g * 3u + 1u] = s1;
  a.grad2d[g * 3u + 2u] = s2;
}

struct StepArgs {
  const gs_frame_data* frames;
  uint32_t n_views, cap, slots;
  float4* P;
  float4* M;
  float4* V;
  float* SH;
  float* MSH;
  float* VSH;
  float4* stats;
  const float4* splat;
  const uint32_t* tiles;
  const float4* grad2d;
  float4* dir_grad;  // per slot: position gradient through the SH view direction (k_step_sh -> k_step_geometry)
  bool view_word;    // grad2d's 12th float holds the view word (ViewBuffers::view_word), not zero
  const uint32_t* d_pairs;
  uint32_t accept;
  Motion motion;  // nodes == 0: no view moves
};

// A (view, slot)'s third grad2d float4 as the pair sums: without the view word.
__device__ __forceinline__ float4 grad_tail(const StepArgs& a, float4 v) {
  if (a.view_word) v.w = 0.0f;
  return v;
}

// Adam (train_step.glsl:62-67). The square root and the division use the hardware's
// approximate forms (PTX sqrt.approx.f32, relative error within 2^-23; div.full.f32,
// within 2 ulp), the precision class of the reference's GLSL sqrt and division; the
// IEEE-rounded sequences cost several times the instructions and a branch each.
__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float div_full(float a, float b) {
  float r;
  asm("div.full.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float adam1(float p, float g, float& m, float& v, float lr, float b1, float b2, float c1,
                                       float c2, float eps) {
  m = g * (1.0f - b1) + m * b1;
  v = g * g * (1.0f - b2) + v * b2;
  return p - lr * div_full(m * c1, sqrt_approx(v * c2) + eps);
}

// Basis function k (1..15) of the real SH basis and its gradient w.r.t. the unit
// direction (train_common.glsl:84-140), one term at a time so unrolled loops keep only
// what they use in registers.
template <int K>
__device__ __forceinline__ float sh_term(float x, float y, float z, float& gx, float& gy, float& gz) {
  constexpr float C1 = 0.4886025119029199f, A = 1.0925484305920792f, B = 0.31539156525252005f,
                  C = 0.5462742152960396f, D = -0.5900435899266435f, E = 2.890611442640554f,
                  F = -0.4570457994644658f, G = 0.3731763325901154f, H = 1.445305721320277f;
  const float xx = x * x, yy = y * y, zz = z * z;
  if constexpr (K == 1) { gx = 0.f; gy = -C1; gz = 0.f; return -C1 * y; }
  if constexpr (K == 2) { gx = 0.f; gy = 0.f; gz = C1; return C1 * z; }
  if constexpr (K == 3) { gx = -C1; gy = 0.f; gz = 0.f; return -C1 * x; }
  if constexpr (K == 4) { gx = A * y; gy = A * x; gz = 0.f; return A * x * y; }
  if constexpr (K == 5) { gx = 0.f; gy = -A * z; gz = -A * y; return -A * y * z; }
  if constexpr (K == 6) { gx = B * (-2.0f * x); gy = B * (-2.0f * y); gz = B * (4.0f * z); return B * (2.0f * zz - xx - yy); }
  if constexpr (K == 7) { gx = -A * z; gy = 0.f; gz = -A * x; return -A * x * z; }
  if constexpr (K == 8) { gx = C * (2.0f * x); gy = C * (-2.0f * y); gz = 0.f; return C * (xx - yy); }
  if constexpr (K == 9) { gx = D * (6.0f * x * y); gy = D * (3.0f * xx - 3.0f * yy); gz = 0.f; return D * y * (3.0f * xx - yy); }
  if constexpr (K == 10) { gx = E * (y * z); gy = E * (x * z); gz = E * (x * y); return E * x * y * z; }
  if constexpr (K == 11) {
    gx = F * (-2.0f * x * y); gy = F * (4.0f * zz - xx - 3.0f * yy); gz = F * (8.0f * y * z);
    return F * y * (4.0f * zz - xx - yy);
  }
  if constexpr (K == 12) {
    gx = G * (-6.0f * x * z); gy = G * (-6.0f * y * z); gz = G * (6.0f * zz - 3.0f * xx - 3.0f * yy);
    return G * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
  }
  if constexpr (K == 13) {
    gx = F * (4.0f * zz - 3.0f * xx - yy); gy = F * (-2.0f * x * y); gz = F * (8.0f * x * z);
    return F * x * (4.0f * zz - xx - yy);
  }
  if constexpr (K == 14) { gx = H * (2.0f * x * z); gy = H * (-2.0f * y * z); gz = H * (xx - yy); return H * z * (xx - yy); }
  if constexpr (K == 15) {
    gx = D * (3.0f * xx - 3.0f * yy); gy = D * (-6.0f * x * y); gz = 0.f;
    return D * x * (xx - 3.0f * yy);
  }
  return 0.0f;
}

template <int... Ks, typename F>
__device__ __forceinline__ void for_terms(std::integer_sequence<int, Ks...>, F&& f) {
  (f(std::integral_constant<int, Ks + 1>{}), ...);
}

// View-independent quantities of a slot's covariance.
// A slot's rotation and scale: M = R S (Sigma = M M^T).
struct Shape {
  float qn[4], qlen, R[3][3], s[3], M[3][3];
};

__device__ __forceinline__ void slot_shape(float4 p1, float4 q, Shape& S) {
  S.qlen = fmaxf(sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w), 1e-12f);
  S.qn[0] = q.x / S.qlen;
  S.qn[1] = q.y / S.qlen;
  S.qn[2] = q.z / S.qlen;
  S.qn[3] = q.w / S.qlen;
  quat_to_matrix(S.qn[0], S.qn[1], S.qn[2], S.qn[3], S.R);
  S.s[0] = expf(p1.x);
  S.s[1] = expf(p1.y);
  S.s[2] = expf(p1.z);
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) S.M[r][c] = S.R[r][c] * S.s[c];
}

// What the per-view backward needs of a slot: its 3D covariance and opacity.
struct Geometry {
  float Sig[3][3], opacity;
};

__device__ __forceinline__ void slot_geometry(float4 p0, float4 p1, float4 q, Geometry& G) {
  Shape S;
  slot_shape(p1, q, S);
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) G.Sig[r][c] = S.M[r][0] * S.M[c][0] + S.M[r][1] * S.M[c][1] + S.M[r][2] * S.M[c][2];
  G.opacity = sigmoidf(p0.w);
}

// The covariance's gradient summed over the views, dSigma (symmetric: 00, 01, 02, 11, 12,
// 22), back to the log scales and the quaternion (train_step.glsl:206-219): dM = 2 dSigma M,
// dL/dlog s_c = s_c sum_r dM_rc R_rc, dL/dR = dM S, then the quaternion's tangent part.
// The map is linear in dSigma, so one pass after the views equals one per view.
__device__ __forceinline__ void scale_rotation_backward(float4 p1, float4 q, const float dsig[6], float g16[16]) {
  Shape S;
  slot_shape(p1, q, S);
  const float dS[3][3] = {{dsig[0], dsig[1], dsig[2]}, {dsig[1], dsig[3], dsig[4]}, {dsig[2], dsig[4], dsig[5]}};
  float dM[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) dM[r][c] = 2.0f * (dS[r][0] * S.M[0][c] + dS[r][1] * S.M[1][c] + dS[r][2] * S.M[2][c]);
#pragma unroll
  for (int c = 0; c < 3; ++c)
    g16[4 + c] += (dM[0][c] * S.R[0][c] + dM[1][c] * S.R[1][c] + dM[2][c] * S.R[2][c]) * S.s[c];
  float gR[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) gR[r][c] = dM[r][c] * S.s[c];
  const float w = S.qn[0], x = S.qn[1], y = S.qn[2], z = S.qn[3];
  float dq[4];
  dq[0] = 2.0f * (-z * gR[0][1] + y * gR[0][2] + z * gR[1][0] - x * gR[1][2] - y * gR[2][0] + x * gR[2][1]);
  dq[1] = 2.0f * (y * gR[0][1] + z * gR[0][2] + y * gR[1][0] - 2.0f * x * gR[1][1] - w * gR[1][2] + z * gR[2][0] +
                  w * gR[2][1] - 2.0f * x * gR[2][2]);
  dq[2] = 2.0f * (-2.0f * y * gR[0][0] + x * gR[0][1] + w * gR[0][2] + x * gR[1][0] + z * gR[1][2] - w * gR[2][0] +
                  z * gR[2][1] - 2.0f * y * gR[2][2]);
  dq[3] = 2.0f * (-2.0f * z * gR[0][0] - w * gR[0][1] + x * gR[0][2] + w * gR[1][0] - 2.0f * z * gR[1][1] +
                  y * gR[1][2] + x * gR[2][0] + y * gR[2][1]);
  const float qd = S.qn[0] * dq[0] + S.qn[1] * dq[1] + S.qn[2] * dq[2] + S.qn[3] * dq[3];
#pragma unroll
  for (int k = 0; k < 4; ++k) g16[8 + k] += (dq[k] - S.qn[k] * qd) / S.qlen;
}

// The views slot i was seen in, as a bit mask: every view's tile count is loaded at once.
__device__ __forceinline__ uint32_t seen_views(const uint32_t* tiles, uint32_t n_views, uint32_t cap, uint32_t i) {
  uint32_t mask = 0u;
#pragma unroll
  for (uint32_t v = 0; v < kMaxViews; ++v)
    if (v < n_views && tiles[size_t(v) * cap + i] != 0u) mask |= 1u << v;
  return mask;
}

// Colour gradient of one view with the clamped channels zeroed (train_step.glsl:135-138).
__device__ __forceinline__ void view_colour_grad(float4 a1, float4 a2, uint32_t clamped, float dcol[3]) {
  dcol[0] = (clamped & 1u) ? 0.0f : a1.z;
  dcol[1] = (clamped & 2u) ? 0.0f : a1.w;
  dcol[2] = (clamped & 4u) ? 0.0f : a2.x;
}

// One view's projection backward (train_step.glsl:82-219) of a slot: adds the gradient of
// the position, opacity and DC parameters to g16 (without the SH view-direction term, which
// k_step_sh computes) and the 3D covariance's gradient to dsig (when non-null; the caller
// takes it to the log scales and the quaternion once, scale_rotation_backward), updates
// the densification statistics, and returns the clamped colour gradient and the view
// direction. drew: bit 0 any pair gradient, bit 1 a non-zero
// colour gradient. With POSE it also adds the slot's share of the camera pose gradient to
// pose (dL/dd, dL/dw; train_step.glsl:196-202).
// With MOTION and dm non-null the slot is moved with the subject in this view
// (train_step.glsl:105-107, 192-194): at dm->x, its covariance turned by dm->U, and the
// position gradient goes back to the rest position through A^T. share (when non-null)
// receives the slot's motion share: dL/dx = V^T dL/dt (world; the SH view-direction term
// is added by the caller) and the turn of its orientation dL/dturn (world axes).
template <int DEG, bool POSE = false, bool MOTION = false>
__device__ __forceinline__ void view_backward(const gs_frame_data& f, float4 p0, const Geometry& G, float4 a0, float4 a1,
                                              float4 a2, uint32_t clamped, float radius, float g16[16], float* dsig,
                                              float4& st,
                                              float dcol[3], float dir[3], float& dir_len, uint32_t& drew,
                                              float* pose = nullptr, const Deformed* dm = nullptr,
                                              float* share = nullptr) {
  if (a0.x != 0.f || a0.y != 0.f || a0.z != 0.f || a0.w != 0.f || a1.x != 0.f || a1.y != 0.f || a1.z != 0.f ||
      a1.w != 0.f || a2.x != 0.f || a2.y != 0.f || a2.z != 0.f || a2.w != 0.f)
    drew |= 1u;
  const float dmx = a0.x, dmy = a0.y;
  const float ga = a0.z, gb = a0.w, gc = a1.x;
  const float dop = a1.y;
  view_colour_grad(a1, a2, clamped, dcol);
  if (dcol[0] != 0.0f || dcol[1] != 0.0f || dcol[2] != 0.0f) drew |= 2u;
  const float width = float(f.image[0]), height = float(f.image[1]);
  const float nx = 0.5f * width, ny = 0.5f * height;
  // Densification statistics: the view-space positional gradient in NDC units.
  st.x += sqrtf((dmx * nx) * (dmx * nx) + (dmy * ny) * (dmy * ny));
  st.y += 1.0f;
  st.z = fmaxf(st.z, radius);
  st.w += sqrtf((a2.y * nx) * (a2.y * nx) + (a2.z * ny) * (a2.z * ny));

  const bool moved = MOTION && dm != nullptr;
  float xm[3] = {p0.x, p0.y, p0.z};  // where the slot is in this view
  // Rest frame -> camera: V, or V U when moved (read from the frame directly without motion).
  float WU[3][3];
  if constexpr (MOTION) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        WU[r][c] = moved ? f.rot[r][0] * dm->U[0][c] + f.rot[r][1] * dm->U[1][c] + f.rot[r][2] * dm->U[2][c]
                         : f.rot[r][c];
    if (moved) {
#pragma unroll
      for (int r = 0; r < 3; ++r) xm[r] = dm->x[r];
    }
  }
  auto W = [&](int r, int c) -> float {
    if constexpr (MOTION) return WU[r][c];
    else return f.rot[r][c];
  };
  float t[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) t[r] = f.rot[r][0] * xm[0] + f.rot[r][1] * xm[1] + f.rot[r][2] * xm[2] + f.rot[r][3];
  const float fx = f.intrinsics[0], fy = f.intrinsics[1], cx = f.intrinsics[2], cy = f.intrinsics[3];
  const float inv_z = 1.0f / t[2];
  const float lim_x = 1.3f * fmaxf(cx, width - cx) / fx;
  const float lim_y = 1.3f * fmaxf(cy, height - cy) / fy;
  const float rx = t[0] * inv_z, ry = t[1] * inv_z;
  const bool clamp_x = rx < -lim_x || rx > lim_x;
  const bool clamp_y = ry < -lim_y || ry > lim_y;
  const float tx = clampf(rx, -lim_x, lim_x), ty = clampf(ry, -lim_y, lim_y);
  const float j00 = fx * inv_z, j02 = -fx * tx * inv_z, j11 = fy * inv_z, j12 = -fy * ty * inv_z;
  float T[2][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    T[0][c] = j00 * W(0, c) + j02 * W(2, c);
    T[1][c] = j11 * W(1, c) + j12 * W(2, c);
  }
  float TS[2][3];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) TS[r][c] = T[r][0] * G.Sig[0][c] + T[r][1] * G.Sig[1][c] + T[r][2] * G.Sig[2][c];
  const float A = TS[0][0] * T[0][0] + TS[0][1] * T[0][1] + TS[0][2] * T[0][2] + kDilation;
  const float B = TS[1][0] * T[0][0] + TS[1][1] * T[0][1] + TS[1][2] * T[0][2];
  const float C = TS[1][0] * T[1][0] + TS[1][1] * T[1][1] + TS[1][2] * T[1][2] + kDilation;
  const float D = A * C - B * B;

  float dr[3] = {xm[0] - f.cam_pos[0], xm[1] - f.cam_pos[1], xm[2] - f.cam_pos[2]};
  if constexpr (MOTION) {
    if (moved) {  // the rest frame's direction, U^T (x - camera)
      const float e[3] = {dr[0], dr[1], dr[2]};
#pragma unroll
      for (int c = 0; c < 3; ++c) dr[c] = dm->U[0][c] * e[0] + dm->U[1][c] * e[1] + dm->U[2][c] * e[2];
    }
  }
  dir_len = fmaxf(sqrtf(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]), 1e-12f);
  dir[0] = dr[0] / dir_len;
  dir[1] = dr[1] / dir_len;
  dir[2] = dr[2] / dir_len;
  g16[12] += 0.28209479177387814f * dcol[0];
  g16[13] += 0.28209479177387814f * dcol[1];
  g16[14] += 0.28209479177387814f * dcol[2];

  g16[3] += dop * G.opacity * (1.0f - G.opacity);

  // Conic -> dilated 2D covariance.
  const float inv_d2 = 1.0f / (D * D);
  const float gA = (-C * C * ga + B * C * gb - B * B * gc) * inv_d2;
  const float gB = (2.0f * B * C * ga - (D + 2.0f * B * B) * gb + 2.0f * A * B * gc) * inv_d2;
  const float gC = (-B * B * ga + A * B * gb - A * A * gc) * inv_d2;
  const float G2[2][2] = {{gA, 0.5f * gB}, {0.5f * gB, gC}};
  // dSigma = T^T G2 T, dT = 2 G2 T Sigma, dJ = dT W^T (J's third row is zero).
  float G2T[2][3];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) G2T[r][c] = G2[r][0] * T[0][c] + G2[r][1] * T[1][c];
  float dT[2][3];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) dT[r][c] = 2.0f * (G2[r][0] * TS[0][c] + G2[r][1] * TS[1][c]);
  float dJ[2][3];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) dJ[r][c] = dT[r][0] * W(c, 0) + dT[r][1] * W(c, 1) + dT[r][2] * W(c, 2);
  float dt[3] = {0.f, 0.f, 0.f};
  const float inv_z2 = inv_z * inv_z;
  dt[2] += -fx * inv_z2 * dJ[0][0] - fy * inv_z2 * dJ[1][1];
  if (clamp_x) {
    dt[2] += fx * tx * inv_z2 * dJ[0][2];
  } else {
    dt[0] += -fx * inv_z2 * dJ[0][2];
    dt[2] += 2.0f * fx * t[0] * inv_z2 * inv_z * dJ[0][2];
  }
  if (clamp_y) {
    dt[2] += fy * ty * inv_z2 * dJ[1][2];
  } else {
    dt[1] += -fy * inv_z2 * dJ[1][2];
    dt[2] += 2.0f * fy * t[1] * inv_z2 * inv_z * dJ[1][2];
  }
  dt[0] += dmx * fx * inv_z;
  dt[1] += dmy * fy * inv_z;
  dt[2] += -(dmx * fx * t[0] + dmy * fy * t[1]) * inv_z2;
  float dx[3];  // dL/dx, world: V^T dL/dt
#pragma unroll
  for (int c = 0; c < 3; ++c) dx[c] = f.rot[0][c] * dt[0] + f.rot[1][c] * dt[1] + f.rot[2][c] * dt[2];
  if constexpr (MOTION) {
    if (moved) {
#pragma unroll
      for (int c = 0; c < 3; ++c) g16[c] += dm->A[0][c] * dx[0] + dm->A[1][c] * dx[1] + dm->A[2][c] * dx[2];
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) g16[c] += dx[c];
    }
    if (share != nullptr) {
      // The orientation's turn in camera axes, (X21 - X12, X02 - X20, X10 - X01) with
      // X = J^T dJ, then in world axes (V^T).
      const float x01 = j00 * dJ[0][1], x02 = j00 * dJ[0][2], x10 = j11 * dJ[1][0], x12 = j11 * dJ[1][2];
      const float x20 = j02 * dJ[0][0] + j12 * dJ[1][0], x21 = j02 * dJ[0][1] + j12 * dJ[1][1];
      const float tc[3] = {x21 - x12, x02 - x20, x10 - x01};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        share[c] = dx[c];
        share[3 + c] = f.rot[0][c] * tc[0] + f.rot[1][c] * tc[1] + f.rot[2][c] * tc[2];
      }
    }
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) g16[c] += dx[c];
  }
  if (POSE) {
    // A shift d moves t by d; a turn w moves t by w x t and W by [w]x W, so with
    // X = dL/dW W^T = J^T dJ: dL/dw = t x dL/dt + (X21 - X12, X02 - X20, X10 - X01).
    const float x01 = j00 * dJ[0][1], x02 = j00 * dJ[0][2], x10 = j11 * dJ[1][0], x12 = j11 * dJ[1][2];
    const float x20 = j02 * dJ[0][0] + j12 * dJ[1][0], x21 = j02 * dJ[0][1] + j12 * dJ[1][1];
    pose[0] += dt[0];
    pose[1] += dt[1];
    pose[2] += dt[2];
    pose[3] += t[1] * dt[2] - t[2] * dt[1] + (x21 - x12);
    pose[4] += t[2] * dt[0] - t[0] * dt[2] + (x02 - x20);
    pose[5] += t[0] * dt[1] - t[1] * dt[0] + (x10 - x01);
  }

  // 3D covariance: dSigma = T^T G2 T, summed over the views (scale_rotation_backward).
  if (dsig != nullptr) {
    dsig[0] += T[0][0] * G2T[0][0] + T[1][0] * G2T[1][0];
    dsig[1] += T[0][0] * G2T[0][1] + T[1][0] * G2T[1][1];
    dsig[2] += T[0][0] * G2T[0][2] + T[1][0] * G2T[1][2];
    dsig[3] += T[0][1] * G2T[0][1] + T[1][1] * G2T[1][1];
    dsig[4] += T[0][1] * G2T[0][2] + T[1][1] * G2T[1][2];
    dsig[5] += T[0][2] * G2T[0][2] + T[1][2] * G2T[1][2];
  }
}

__device__ __forceinline__ void adam_params(const StepArgs& a, const gs_frame_data& f0, uint32_t i, float4 p0,
                                            float4 p1, float4 q, float4 p3, const float g16[16]) {
  const float b1 = f0.adam[0], b2 = f0.adam[1], eps = f0.adam[2], c1 = f0.bias[0], c2 = f0.bias[1];
  float4 m0 = a.M[i], m1 = a.M[a.cap + i], m2 = a.M[2u * a.cap + i], m3 = a.M[3u * a.cap + i];
  float4 v0 = a.V[i], v1 = a.V[a.cap + i], v2 = a.V[2u * a.cap + i], v3 = a.V[3u * a.cap + i];
  const float lp = f0.lr0[0], ls = f0.lr0[1], lq = f0.lr0[2], lo = f0.lr0[3], ld = f0.lr1[0];
  p0.x = adam1(p0.x, g16[0], m0.x, v0.x, lp, b1, b2, c1, c2, eps);
  p0.y = adam1(p0.y, g16[1], m0.y, v0.y, lp, b1, b2, c1, c2, eps);
  p0.z = adam1(p0.z, g16[2], m0.z, v0.z, lp, b1, b2, c1, c2, eps);
  p0.w = adam1(p0.w, g16[3], m0.w, v0.w, lo, b1, b2, c1, c2, eps);
  p1.x = adam1(p1.x, g16[4], m1.x, v1.x, ls, b1, b2, c1, c2, eps);
  p1.y = adam1(p1.y, g16[5], m1.y, v1.y, ls, b1, b2, c1, c2, eps);
  p1.z = adam1(p1.z, g16[6], m1.z, v1.z, ls, b1, b2, c1, c2, eps);
  p1.w = adam1(p1.w, 0.0f, m1.w, v1.w, 0.0f, b1, b2, c1, c2, eps);
  q.x = adam1(q.x, g16[8], m2.x, v2.x, lq, b1, b2, c1, c2, eps);
  q.y = adam1(q.y, g16[9], m2.y, v2.y, lq, b1, b2, c1, c2, eps);
  q.z = adam1(q.z, g16[10], m2.z, v2.z, lq, b1, b2, c1, c2, eps);
  q.w = adam1(q.w, g16[11], m2.w, v2.w, lq, b1, b2, c1, c2, eps);
  p3.x = adam1(p3.x, g16[12], m3.x, v3.x, ld, b1, b2, c1, c2, eps);
  p3.y = adam1(p3.y, g16[13], m3.y, v3.y, ld, b1, b2, c1, c2, eps);
  p3.z = adam1(p3.z, g16[14], m3.z, v3.z, ld, b1, b2, c1, c2, eps);
  p3.w = adam1(p3.w, 0.0f, m3.w, v3.w, 0.0f, b1, b2, c1, c2, eps);
  a.P[i] = p0;
  a.P[a.cap + i] = p1;
  a.P[2u * a.cap + i] = q;
  a.P[3u * a.cap + i] = p3;
  a.M[i] = m0;
  a.M[a.cap + i] = m1;
  a.M[2u * a.cap + i] = m2;
  a.M[3u * a.cap + i] = m3;
  a.V[i] = v0;
  a.V[a.cap + i] = v1;
  a.V[2u * a.cap + i] = v2;
  a.V[3u * a.cap + i] = v3;
}

__device__ __forceinline__ void copy_frames(const StepArgs& a, gs_frame_data* s_frames, uint32_t n) {
  const uint32_t words = n * uint32_t(sizeof(gs_frame_data) / 4);
  for (uint32_t k = threadIdx.x; k < words; k += blockDim.x)
    reinterpret_cast<uint32_t*>(s_frames)[k] = reinterpret_cast<const uint32_t*>(a.frames)[k];
  __syncthreads();
}

// Part 1 (train_step_sh.comp:21-44 and the SH view-direction term of
// train_step.glsl:131-155): one thread per slot. The slot's SH coefficients are loaded
// once; for each view the slot was seen in, the basis and its direction gradient are
// evaluated once, giving all 3K coefficient gradients (added in view order) and dL/d(dir),
// which goes through the normalisation into the position gradient (summed over views,
// stored for part 2). Then Adam on the 3K coefficients, 3 coefficients' moments loaded
// together so each thread keeps 18 loads in flight (the SH values are already loaded).
// Capped at 128 registers (4 blocks per SM, a few spills): 55 us faster on 8 views of 1M
// slots than 3 blocks at 168 registers; at 5 blocks (96 registers) the spills cost more.
template <int DEG, bool MOTION, bool WORD>
__global__ void __launch_bounds__(128, 4) k_step_sh(StepArgs a) {
  __shared__ gs_frame_data s_frames[kMaxViews];
  copy_frames(a, s_frames, a.n_views);
  if (*a.d_pairs > a.accept) return;
  constexpr int K = DEG == 0 ? 0 : (DEG + 1) * (DEG + 1) - 1;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.slots) return;
  const float4 p0 = a.P[i];
  if (a.P[a.cap + i].w < 0.5f) return;
  float sh[K][3];
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) sh[k][c] = a.SH[size_t(3 * k + c) * a.cap + i];
  float g[K][3];
#pragma unroll
  for (int k = 0; k < K; ++k) g[k][0] = g[k][1] = g[k][2] = 0.0f;
  float pd[3] = {0.f, 0.f, 0.f};
  bool colour = false;
  // Views in order; the next view's loads are issued before this view's arithmetic.
  uint32_t mask = seen_views(a.tiles, a.n_views, a.cap, i);
  uint32_t nv = mask ? uint32_t(__ffs(mask) - 1) : 0u;
  float4 n1 = make_float4(0.f, 0.f, 0.f, 0.f), n2 = n1;
  float nw = 0.0f;
  if (mask) {
    const size_t gv = size_t(nv) * a.cap + i;
    n1 = a.grad2d[gv * 3u + 1u];
    n2 = a.grad2d[gv * 3u + 2u];
    if (!WORD) nw = a.splat[gv * 3u + 2u].w;
  }
  while (mask) {
    const uint32_t v = nv;
    const float4 a1 = n1, a2 = n2;
    const float cw = nw;
    mask &= mask - 1u;
    if (mask) {
      nv = uint32_t(__ffs(mask) - 1);
      const size_t gv = size_t(nv) * a.cap + i;
      n1 = a.grad2d[gv * 3u + 1u];
      n2 = a.grad2d[gv * 3u + 2u];
      if (!WORD) nw = a.splat[gv * 3u + 2u].w;
    }
    float dcol[3];
    view_colour_grad(a1, a2, WORD ? view_word_clamped(a2.w) : __float_as_uint(cw), dcol);
    colour |= dcol[0] != 0.0f || dcol[1] != 0.0f || dcol[2] != 0.0f;
    const gs_frame_data& f = s_frames[v];
    float dr[3] = {p0.x - f.cam_pos[0], p0.y - f.cam_pos[1], p0.z - f.cam_pos[2]};
    Deformed dm;
    bool moved = false;
    if constexpr (MOTION) {
      if ((f.model[3] & GS_FLAG_MOTION) != 0u) {  // the rest frame's direction, U^T (x - camera)
        deform(a.motion, a.motion.views + size_t(v) * kMaxMotionNodes, i, p0.x, p0.y, p0.z, dm);
        const float e[3] = {dm.x[0] - f.cam_pos[0], dm.x[1] - f.cam_pos[1], dm.x[2] - f.cam_pos[2]};
#pragma unroll
        for (int c = 0; c < 3; ++c) dr[c] = dm.U[0][c] * e[0] + dm.U[1][c] * e[1] + dm.U[2][c] * e[2];
        moved = true;
      }
    }
    const float dir_len = fmaxf(sqrtf(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]), 1e-12f);
    const float dir[3] = {dr[0] / dir_len, dr[1] / dir_len, dr[2] / dir_len};
    float dd[3] = {0.f, 0.f, 0.f};
    for_terms(std::make_integer_sequence<int, K>{}, [&](auto kk) {
      constexpr int k = decltype(kk)::value;
      float gx, gy, gz;
      const float b = sh_term<k>(dir[0], dir[1], dir[2], gx, gy, gz);
#pragma unroll
      for (int c = 0; c < 3; ++c) g[k - 1][c] += b * dcol[c];
      const float w = sh[k - 1][0] * dcol[0] + sh[k - 1][1] * dcol[1] + sh[k - 1][2] * dcol[2];
      dd[0] += w * gx;
      dd[1] += w * gy;
      dd[2] += w * gz;
    });
    const float proj = dir[0] * dd[0] + dir[1] * dd[1] + dir[2] * dd[2];
    if constexpr (MOTION) {
      if (moved) {  // back through U to x, then through A^T to the rest position
        float gd[3], gx[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) gd[c] = (dd[c] - dir[c] * proj) / dir_len;
#pragma unroll
        for (int r = 0; r < 3; ++r) gx[r] = dm.U[r][0] * gd[0] + dm.U[r][1] * gd[1] + dm.U[r][2] * gd[2];
#pragma unroll
        for (int c = 0; c < 3; ++c) pd[c] += dm.A[0][c] * gx[0] + dm.A[1][c] * gx[1] + dm.A[2][c] * gx[2];
        continue;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) pd[c] += (dd[c] - dir[c] * proj) / dir_len;
  }
  a.dir_grad[i] = make_float4(pd[0], pd[1], pd[2], 0.0f);
  const gs_frame_data& f0 = s_frames[0];
  if ((f0.model[3] & GS_FLAG_SPARSE_ADAM) != 0u && !colour) return;
  const float b1 = f0.adam[0], b2 = f0.adam[1], eps = f0.adam[2], c1 = f0.bias[0], c2 = f0.bias[1], lr = f0.lr1[1];
  constexpr int kChunk = 3;
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += kChunk) {
    float m[kChunk][3], v[kChunk][3];
#pragma unroll
    for (int j = 0; j < kChunk; ++j)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (k0 + j < K) {
          const size_t o = size_t(3 * (k0 + j) + c) * a.cap + i;
          m[j][c] = a.MSH[o];
          v[j][c] = a.VSH[o];
        }
#pragma unroll
    for (int j = 0; j < kChunk; ++j)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (k0 + j < K) {
          const size_t o = size_t(3 * (k0 + j) + c) * a.cap + i;
          a.SH[o] = adam1(sh[k0 + j][c], g[k0 + j][c], m[j][c], v[j][c], lr, b1, b2, c1, c2, eps);
          a.MSH[o] = m[j][c];
          a.VSH[o] = v[j][c];
        }
  }
}

// Part 2 (train_step.glsl:72-240): every view's projection backward summed, plus the SH
// view-direction term from part 1, then Adam on the 16 parameters.
template <int DEG, bool MOTION, bool WORD>
__global__ void __launch_bounds__(128, 5) k_step_geometry(StepArgs a) {
  __shared__ gs_frame_data s_frames[kMaxViews];
  copy_frames(a, s_frames, a.n_views);
  if (*a.d_pairs > a.accept) return;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.slots) return;
  const float4 p0 = a.P[i], p1 = a.P[a.cap + i], q = a.P[2u * a.cap + i], p3 = a.P[3u * a.cap + i];
  if (p1.w < 0.5f) return;
  float g16[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) g16[k] = 0.0f;
  uint32_t drew = 0u;
  Geometry G;
  slot_geometry(p0, p1, q, G);
  float dsig[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float4 st = a.stats[i];
  // Views in order; the next view's loads are issued before this view's arithmetic.
  uint32_t mask = seen_views(a.tiles, a.n_views, a.cap, i);
  const bool seen = mask != 0u;
  uint32_t nv = mask ? uint32_t(__ffs(mask) - 1) : 0u;
  float4 n0 = make_float4(0.f, 0.f, 0.f, 0.f), n1 = n0, n2 = n0;
  float nw = 0.0f, nr = 0.0f;
  if (mask) {
    const size_t g = size_t(nv) * a.cap + i;
    n0 = a.grad2d[g * 3u];
    n1 = a.grad2d[g * 3u + 1u];
    n2 = a.grad2d[g * 3u + 2u];
    if (!WORD) {
      nw = a.splat[g * 3u + 2u].w;
      nr = a.splat[g * 3u + 1u].w;
    }
  }
  while (mask) {
    const uint32_t v = nv;
    const float4 a0 = n0, a1 = n1, a2 = WORD ? make_float4(n2.x, n2.y, n2.z, 0.0f) : n2;
    const float cw = WORD ? __uint_as_float(view_word_clamped(n2.w)) : nw;
    const float radius = WORD ? view_word_radius(n2.w) : nr;
    mask &= mask - 1u;
    if (mask) {
      nv = uint32_t(__ffs(mask) - 1);
      const size_t g = size_t(nv) * a.cap + i;
      n0 = a.grad2d[g * 3u];
      n1 = a.grad2d[g * 3u + 1u];
      n2 = a.grad2d[g * 3u + 2u];
      if (!WORD) {
        nw = a.splat[g * 3u + 2u].w;
        nr = a.splat[g * 3u + 1u].w;
      }
    }
    float dcol[3], dir[3], dir_len;
    if constexpr (MOTION) {
      if ((s_frames[v].model[3] & GS_FLAG_MOTION) != 0u) {
        Deformed dm;
        deform(a.motion, a.motion.views + size_t(v) * kMaxMotionNodes, i, p0.x, p0.y, p0.z, dm);
        view_backward<DEG, false, true>(s_frames[v], p0, G, a0, a1, a2, __float_as_uint(cw), radius, g16, dsig, st,
                                        dcol, dir, dir_len, drew, nullptr, &dm);
        continue;
      }
    }
    view_backward<DEG>(s_frames[v], p0, G, a0, a1, a2, __float_as_uint(cw), radius, g16, dsig, st, dcol, dir, dir_len,
                       drew);
  }
  if (DEG > 0) {
    const float4 pd = a.dir_grad[i];
    g16[0] += pd.x;
    g16[1] += pd.y;
    g16[2] += pd.z;
  }
  if (seen) {
    scale_rotation_backward(p1, q, dsig, g16);
    a.stats[i] = st;
  }
  const gs_frame_data& f0 = s_frames[0];
  const bool sparse = (f0.model[3] & GS_FLAG_SPARSE_ADAM) != 0u;
  if (!sparse || (drew & 1u)) adam_params(a, f0, i, p0, p1, q, p3, g16);
}

// Camera pose gradient (train_step.glsl:196-202, 254-268): block (x, v) sums the shares of
// its 128 slots in view v, if that view asks for it, in a fixed order (a butterfly per
// warp, then the warps) into partial[(v * gridDim.x + x) * 8 + 0..5]. Parameters are read
// before the step's update, as in the reference's single pass; the SH view-direction term
// is left out there too.
template <int DEG, bool MOTION>
__global__ void __launch_bounds__(128) k_pose_grad(StepArgs a, float* __restrict__ partial) {
  __shared__ gs_frame_data s_frame;
  __shared__ float s_red[4][6];
  const uint32_t v = blockIdx.y;
  if (threadIdx.x < uint32_t(sizeof(gs_frame_data) / 4))
    reinterpret_cast<uint32_t*>(&s_frame)[threadIdx.x] = reinterpret_cast<const uint32_t*>(a.frames + v)[threadIdx.x];
  __syncthreads();
  if ((s_frame.model[3] & GS_FLAG_POSE_GRAD) == 0u) return;  // the whole block
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  float pose[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (i < a.slots && *a.d_pairs <= a.accept) {
    const size_t g = size_t(v) * a.cap + i;
    const float4 p1 = a.P[a.cap + i];
    if (p1.w >= 0.5f && a.tiles[g] != 0u) {
      const float4 p0 = a.P[i], q = a.P[2u * a.cap + i];
      Geometry G;
      slot_geometry(p0, p1, q, G);
      float g16[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) g16[k] = 0.0f;
      float4 st = make_float4(0.f, 0.f, 0.f, 0.f);
      float dcol[3], dir[3], dir_len;
      uint32_t drew = 0u;
      const float4 a0 = a.grad2d[g * 3u], a1 = a.grad2d[g * 3u + 1u], a2 = grad_tail(a, a.grad2d[g * 3u + 2u]);
      const uint32_t clamped = __float_as_uint(a.splat[g * 3u + 2u].w);
      bool done = false;
      if constexpr (MOTION) {
        if ((s_frame.model[3] & GS_FLAG_MOTION) != 0u) {
          Deformed dm;
          deform(a.motion, a.motion.views + size_t(v) * kMaxMotionNodes, i, p0.x, p0.y, p0.z, dm);
          view_backward<DEG, true, true>(s_frame, p0, G, a0, a1, a2, clamped, 0.0f, g16, nullptr, st, dcol, dir, dir_len,
                                         drew, pose, &dm);
          done = true;
        }
      }
      if (!done)
        view_backward<DEG, true>(s_frame, p0, G, a0, a1, a2, clamped, 0.0f, g16, nullptr, st, dcol, dir, dir_len, drew,
                                 pose);
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pose[k] += __shfl_xor_sync(0xffffffffu, pose[k], o);
  if ((threadIdx.x & 31u) == 0u)
#pragma unroll
    for (int k = 0; k < 6; ++k) s_red[threadIdx.x >> 5][k] = pose[k];
  __syncthreads();
  if (threadIdx.x < 6u)
    partial[(size_t(v) * gridDim.x + blockIdx.x) * 8u + threadIdx.x] =
        ((s_red[0][threadIdx.x] + s_red[1][threadIdx.x]) + s_red[2][threadIdx.x]) + s_red[3][threadIdx.x];
}

// The blocks' pose sums per view, in double and a fixed order (Trainer::pose_gradient,
// trainer.cpp:1336-1348), into out[v * stride + 0..5]; 0 for views without the flag.
__global__ void __launch_bounds__(256) k_pose_reduce(const gs_frame_data* frames, const float* __restrict__ partial,
                                                     uint32_t blocks, double* __restrict__ out, uint32_t stride) {
  __shared__ double s[8][6];
  const uint32_t v = blockIdx.x;
  const bool wanted = (frames[v].model[3] & GS_FLAG_POSE_GRAD) != 0u;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  if (wanted)
    for (uint32_t b = threadIdx.x; b < blocks; b += 256u)
#pragma unroll
      for (int k = 0; k < 6; ++k) acc[k] += double(partial[(size_t(v) * blocks + b) * 8u + k]);
#pragma unroll
  for (int k = 0; k < 6; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if ((threadIdx.x & 31u) == 0u)
#pragma unroll
    for (int k = 0; k < 6; ++k) s[threadIdx.x >> 5][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < 6u) {
    double sum = 0.0;
    for (int w = 0; w < 8; ++w) sum += s[w][threadIdx.x];
    out[size_t(v) * stride + threadIdx.x] = sum;
  }
}

// ---- subject motion ----

// The motion gradient (train_step.glsl:270-337 with train_motion_sum.comp) of view
// blockIdx.y, if it has GS_FLAG_MOTION_GRAD: per node k, over the slots that follow it,
//   dL/dshift_k = sum w_k dL/dx,   dL/dturn_k = sum w_k (tau + (R_k (p - n_k)) x dL/dx),
// with dL/dx the slot's moved-position gradient (world, including the SH view-direction
// term) and tau the turn of its orientation. Blocks walk chunks of 128 slots; a chunk's
// nodes are listed, the threads split between them (a power of two per node, up to 16),
// each part sums a slice of the chunk in slot order, and each node adds its parts in order
// to the block's total: a fixed summation order for a fixed grid. The block writes its
// totals to partial[((v * gridDim.x + block) * kMaxMotionNodes + node) * 8 + 0..5].
template <int DEG>
__global__ void __launch_bounds__(128) k_motion_grad(StepArgs a, float* __restrict__ partial) {
  constexpr int K = DEG == 0 ? 0 : (DEG + 1) * (DEG + 1) - 1;
  __shared__ gs_frame_data s_frame;
  __shared__ float s_rest[3][128];
  __shared__ float s_share[6][128];
  __shared__ uint4 s_nodes[128];
  __shared__ float4 s_w[128];
  __shared__ uint32_t s_mask[4];
  __shared__ uint32_t s_list[128];
  __shared__ float s_part[6][128];
  __shared__ float s_acc[6][kMaxMotionNodes];
  const uint32_t v = blockIdx.y, l = threadIdx.x;
  if (l < uint32_t(sizeof(gs_frame_data) / 4))
    reinterpret_cast<uint32_t*>(&s_frame)[l] = reinterpret_cast<const uint32_t*>(a.frames + v)[l];
  for (uint32_t k = l; k < 6u * kMaxMotionNodes; k += 128u) (&s_acc[0][0])[k] = 0.0f;
  __syncthreads();
  if ((s_frame.model[3] & GS_FLAG_MOTION_GRAD) == 0u) return;  // the whole block
  const uint32_t n_nodes = min(a.motion.nodes, kMaxMotionNodes);
  const MotionNode* table = a.motion.views + size_t(v) * kMaxMotionNodes;
  const bool moving = (s_frame.model[3] & GS_FLAG_MOTION) != 0u;
  const bool valid = *a.d_pairs <= a.accept;
  for (uint32_t base = blockIdx.x * 128u; base < a.slots; base += gridDim.x * 128u) {
    const uint32_t i = base + l;
    float share[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f);
    uint4 nodes = make_uint4(0u, 0u, 0u, 0u), wbits = nodes;
    bool any = false;
    if (valid && i < a.slots) {
      const size_t g = size_t(v) * a.cap + i;
      const float4 p1 = a.P[a.cap + i];
      if (p1.w >= 0.5f && a.tiles[g] != 0u) {
        p0 = a.P[i];
        Geometry G;
        slot_geometry(p0, p1, a.P[2u * a.cap + i], G);
        Deformed dm;
        if (moving) deform(a.motion, table, i, p0.x, p0.y, p0.z, dm);
        else at_rest(p0.x, p0.y, p0.z, dm);
        float g16[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) g16[k] = 0.0f;
        float4 st = make_float4(0.f, 0.f, 0.f, 0.f);
        float dcol[3], dir[3], dir_len;
        uint32_t drew = 0u;
        view_backward<DEG, false, true>(s_frame, p0, G, a.grad2d[g * 3u], a.grad2d[g * 3u + 1u],
                                        grad_tail(a, a.grad2d[g * 3u + 2u]), __float_as_uint(a.splat[g * 3u + 2u].w),
                                        0.0f, g16, nullptr, st, dcol, dir, dir_len, drew, nullptr, &dm, share);
        if constexpr (K > 0) {
          // The SH view-direction term of dL/dx: U (dd - dir (dir . dd)) / |x - c|.
          float dd[3] = {0.f, 0.f, 0.f};
          for_terms(std::make_integer_sequence<int, K>{}, [&](auto kk) {
            constexpr int k = decltype(kk)::value;
            float gx, gy, gz;
            sh_term<k>(dir[0], dir[1], dir[2], gx, gy, gz);
            const float w = a.SH[size_t(3 * (k - 1)) * a.cap + i] * dcol[0] +
                            a.SH[size_t(3 * (k - 1) + 1) * a.cap + i] * dcol[1] +
                            a.SH[size_t(3 * (k - 1) + 2) * a.cap + i] * dcol[2];
            dd[0] += w * gx;
            dd[1] += w * gy;
            dd[2] += w * gz;
          });
          const float proj = dir[0] * dd[0] + dir[1] * dd[1] + dir[2] * dd[2];
          float gd[3];
#pragma unroll
          for (int c = 0; c < 3; ++c) gd[c] = (dd[c] - dir[c] * proj) / dir_len;
#pragma unroll
          for (int r = 0; r < 3; ++r) share[r] += dm.U[r][0] * gd[0] + dm.U[r][1] * gd[1] + dm.U[r][2] * gd[2];
        }
        nodes = a.motion.bind[2u * i];
        wbits = a.motion.bind[2u * i + 1u];
        any = true;
      }
    }
    s_rest[0][l] = p0.x;
    s_rest[1][l] = p0.y;
    s_rest[2][l] = p0.z;
#pragma unroll
    for (int k = 0; k < 6; ++k) s_share[k][l] = share[k];
    s_nodes[l] = nodes;
    s_w[l] = any ? make_float4(__uint_as_float(wbits.x), __uint_as_float(wbits.y), __uint_as_float(wbits.z),
                               __uint_as_float(wbits.w))
                 : make_float4(0.f, 0.f, 0.f, 0.f);
    if (l < 4u) s_mask[l] = 0u;
    __syncthreads();
    if (any) {
      const uint32_t nk[4] = {nodes.x, nodes.y, nodes.z, nodes.w};
      const float wk[4] = {__uint_as_float(wbits.x), __uint_as_float(wbits.y), __uint_as_float(wbits.z),
                           __uint_as_float(wbits.w)};
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (wk[j] != 0.0f && nk[j] < n_nodes) atomicOr(&s_mask[nk[j] >> 5], 1u << (nk[j] & 31u));
    }
    __syncthreads();
    const uint32_t word = l >> 5, bit = 1u << (l & 31u);
    const bool mine = l < n_nodes && (s_mask[word] & bit) != 0u;
    uint32_t place = __popc(s_mask[word] & (bit - 1u)), count = 0u;
#pragma unroll
    for (uint32_t w4 = 0; w4 < 4u; ++w4) {
      const uint32_t c = __popc(s_mask[w4]);
      count += c;
      if (w4 < word) place += c;
    }
    if (mine) s_list[place] = l;
    const uint32_t parts = count <= 1u ? 16u : min(16u, 128u >> (32u - __clz(count - 1u)));
    const uint32_t per = 128u / parts;
    __syncthreads();
    float part[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (l < count * parts) {
      const uint32_t node = s_list[l / parts], first = (l % parts) * per;
      const MotionNode& n = table[node];
      for (uint32_t j = first; j < first + per; ++j) {
        const uint4 nj = s_nodes[j];
        const float4 wj = s_w[j];
        const float wl = nj.x == node ? wj.x : nj.y == node ? wj.y : nj.z == node ? wj.z : nj.w == node ? wj.w : 0.0f;
        if (wl == 0.0f) continue;
        const float px = s_rest[0][j], py = s_rest[1][j], pz = s_rest[2][j];
        // The arm R_k (p - n_k) = R_k p + b_k - c_k.
        const float arm[3] = {n.row[0].x * px + n.row[0].y * py + n.row[0].z * pz + n.row[0].w - n.moved.x,
                              n.row[1].x * px + n.row[1].y * py + n.row[1].z * pz + n.row[1].w - n.moved.y,
                              n.row[2].x * px + n.row[2].y * py + n.row[2].z * pz + n.row[2].w - n.moved.z};
        const float d[3] = {s_share[0][j], s_share[1][j], s_share[2][j]};
        part[0] += wl * d[0];
        part[1] += wl * d[1];
        part[2] += wl * d[2];
        part[3] += wl * (s_share[3][j] + (arm[1] * d[2] - arm[2] * d[1]));
        part[4] += wl * (s_share[4][j] + (arm[2] * d[0] - arm[0] * d[2]));
        part[5] += wl * (s_share[5][j] + (arm[0] * d[1] - arm[1] * d[0]));
      }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) s_part[k][l] = part[k];
    __syncthreads();
    if (mine) {
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        float sum = 0.0f;
        for (uint32_t q = place * parts; q < (place + 1u) * parts; ++q) sum += s_part[k][q];
        s_acc[k][l] += sum;
      }
    }
    __syncthreads();
  }
  if (l < n_nodes) {
    float* out = partial + ((size_t(v) * gridDim.x + blockIdx.x) * kMaxMotionNodes + l) * 8u;
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = s_acc[k][l];
  }
}

// Per view and node: the blocks' motion sums in double, in block order, into
// out[(v * kMaxMotionNodes + node) * 8 + 0..5]; 0 for views without GS_FLAG_MOTION_GRAD.
__global__ void __launch_bounds__(64) k_motion_reduce(const gs_frame_data* frames, const float* __restrict__ partial,
                                                      uint32_t blocks, double* __restrict__ out) {
  __shared__ double s[2][6];
  const uint32_t node = blockIdx.x, v = blockIdx.y;
  const bool wanted = (frames[v].model[3] & GS_FLAG_MOTION_GRAD) != 0u;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  if (wanted)
    for (uint32_t b = threadIdx.x; b < blocks; b += 64u) {
      const float* p = partial + ((size_t(v) * blocks + b) * kMaxMotionNodes + node) * 8u;
#pragma unroll
      for (int k = 0; k < 6; ++k) acc[k] += double(p[k]);
    }
#pragma unroll
  for (int k = 0; k < 6; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if ((threadIdx.x & 31u) == 0u)
#pragma unroll
    for (int k = 0; k < 6; ++k) s[threadIdx.x >> 5][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < 6u) out[(size_t(v) * kMaxMotionNodes + node) * 8u + threadIdx.x] = s[0][threadIdx.x] + s[1][threadIdx.x];
}

// train_motion_bind.comp: each slot in use to its 4 nearest nodes at its rest position
// (ties keep the lower node), weights exp(-d^2 / (2 r^2)) normalised, the nearest alone
// when they all underflow; free slots get no nodes.
__global__ void __launch_bounds__(128) k_motion_bind(const float4* __restrict__ P, uint32_t cap, uint32_t slots,
                                                     const float4* __restrict__ rest, uint32_t n_nodes,
                                                     uint4* __restrict__ bind) {
  __shared__ float4 s_rest[kMaxMotionNodes];
  for (uint32_t k = threadIdx.x; k < n_nodes; k += blockDim.x) s_rest[k] = rest[k];
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= slots) return;
  uint32_t best[4] = {0u, 0u, 0u, 0u};
  float dist[4] = {1e30f, 1e30f, 1e30f, 1e30f};
  if (P[cap + i].w > 0.5f) {
    const float4 p = P[i];
    for (uint32_t k = 0; k < n_nodes; ++k) {
      const float dx = p.x - s_rest[k].x, dy = p.y - s_rest[k].y, dz = p.z - s_rest[k].z;
      const float d2 = dx * dx + dy * dy + dz * dz;
      if (!(d2 < dist[3])) continue;
      // Insert into the sorted four (strictly nearer moves ahead).
      int j = 3;
      while (j > 0 && d2 < dist[j - 1]) {
        dist[j] = dist[j - 1];
        best[j] = best[j - 1];
        --j;
      }
      dist[j] = d2;
      best[j] = k;
    }
  }
  float w[4] = {0.f, 0.f, 0.f, 0.f}, sum = 0.0f;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (dist[j] >= 1e30f) continue;
    w[j] = expf(-dist[j] * s_rest[best[j]].w);
    sum += w[j];
  }
  if (sum > 1e-20f) {
#pragma unroll
    for (int j = 0; j < 4; ++j) w[j] /= sum;
  } else if (dist[0] < 1e30f) {
    w[0] = 1.0f;  // far from every node: the nearest alone
    w[1] = w[2] = w[3] = 0.0f;
  }
  bind[2u * i] = make_uint4(best[0], best[1], best[2], best[3]);
  bind[2u * i + 1u] = make_uint4(__float_as_uint(w[0]), __float_as_uint(w[1]), __float_as_uint(w[2]),
                                 __float_as_uint(w[3]));
}

// ---- densification ----

struct DensifyArgs {
  const gs_frame_data* frame;
  uint32_t cap, slots, sh_stride;
  float4* P;
  float4* M;
  float4* V;
  float* SH;
  float* MSH;
  float* VSH;
  const float4* stats;
  uint32_t* spawn;
  uint32_t* release;
  uint32_t* wants;
  const uint32_t* free_pos;
  const uint32_t* spawn_pos;
  uint32_t* free_list;
  uint32_t* counters;
};

__device__ __forceinline__ void clear_moments(const DensifyArgs& a, uint32_t slot) {
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    a.M[size_t(k) * a.cap + slot] = z;
    a.V[size_t(k) * a.cap + slot] = z;
  }
  for (uint32_t k = 0; k < a.sh_stride; ++k) {
    a.MSH[size_t(k) * a.cap + slot] = 0.0f;
    a.VSH[size_t(k) * a.cap + slot] = 0.0f;
  }
}

// train_densify_mark.comp:22-57
__global__ void __launch_bounds__(128) k_densify_mark(DensifyArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.slots) return;
  const gs_frame_data& f = *a.frame;
  const float4 p0 = a.P[i], p1 = a.P[a.cap + i];
  uint32_t action = 0u;
  bool release = p1.w < 0.5f;
  if (!release) {
    const float4 st = a.stats[i];
    const float max_scale = expf(fmaxf(p1.x, fmaxf(p1.y, p1.z)));
    bool prune = sigmoidf(p0.w) < f.densify0[2];
    if (f.densify0[3] > 0.0f && max_scale > f.densify0[3]) prune = true;
    if (f.densify1[0] > 0.0f && st.z > f.densify1[0]) prune = true;
    if (prune) {
      release = true;
      atomicAdd(&a.counters[2], 1u);
      a.P[i] = make_float4(0.f, 0.f, 0.f, -20.0f);
      a.P[a.cap + i] = make_float4(0.f, 0.f, 0.f, 0.f);
      a.P[2u * a.cap + i] = make_float4(1.f, 0.f, 0.f, 0.f);
      a.P[3u * a.cap + i] = make_float4(0.f, 0.f, 0.f, 0.f);
      for (uint32_t k = 0; k < a.sh_stride; ++k) a.SH[size_t(k) * a.cap + i] = 0.0f;
      clear_moments(a, i);
    } else if (st.y > 0.0f && st.x / st.y >= f.densify0[0]) {
      action = max_scale <= f.densify0[1] ? 1u : 2u;
    }
  }
  a.spawn[i] = action;
  a.release[i] = release ? 1u : 0u;
  a.wants[i] = action != 0u ? 1u : 0u;
}

__global__ void __launch_bounds__(128) k_free_list(DensifyArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.slots) return;
  if (a.release[i]) a.free_list[a.free_pos[i]] = i;
}

// PCG hash and normal sample of train_common.glsl:145-161.
__device__ __forceinline__ uint32_t pcg_hash(uint32_t v) {
  const uint32_t state = v * 747796405u + 2891336453u;
  const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}
__device__ __forceinline__ float uniform01(uint32_t& state) {
  state = pcg_hash(state);
  return float(state >> 8u) * (1.0f / 16777216.0f);
}
__device__ __forceinline__ void normal3(uint32_t& state, float out[3]) {
  const float u1 = fmaxf(uniform01(state), 1e-7f), u2 = uniform01(state);
  const float u3 = fmaxf(uniform01(state), 1e-7f), u4 = uniform01(state);
  const float r1 = sqrtf(-2.0f * logf(u1)), r2 = sqrtf(-2.0f * logf(u3));
  out[0] = r1 * cosf(6.283185307f * u2);
  out[1] = r1 * sinf(6.283185307f * u2);
  out[2] = r2 * cosf(6.283185307f * u4);
}

// train_densify_spawn.comp:38-70, the k-th spawner in slot order taking the k-th free slot.
__global__ void __launch_bounds__(128) k_densify_spawn(DensifyArgs a, uint32_t capacity) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.slots) return;
  const uint32_t action = a.spawn[i];
  if (action == 0u) return;
  const gs_frame_data& f = *a.frame;
  const uint32_t k = a.spawn_pos[i];
  const uint32_t free_count = a.counters[0];
  const uint32_t target = k < free_count ? a.free_list[k] : a.slots + (k - free_count);
  if (target >= capacity) return;
  const float4 p0 = a.P[i], p1 = a.P[a.cap + i], q = a.P[2u * a.cap + i], p3 = a.P[3u * a.cap + i];
  for (uint32_t c = 0; c < a.sh_stride; ++c) a.SH[size_t(c) * a.cap + target] = a.SH[size_t(c) * a.cap + i];
  clear_moments(a, target);
  if (action == 1u) {
    a.P[target] = p0;
    a.P[a.cap + target] = p1;
  } else {
    uint32_t seed_bits;
    memcpy(&seed_bits, &f.densify1[1], 4);
    uint32_t rng = pcg_hash(i ^ pcg_hash(seed_bits));
    const float s[3] = {expf(p1.x), expf(p1.y), expf(p1.z)};
    const float qlen = fmaxf(sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w), 1e-12f);
    float R[3][3];
    quat_to_matrix(q.x / qlen, q.y / qlen, q.z / qlen, q.w / qlen, R);
    float na[3], nb[3];
    normal3(rng, na);
    normal3(rng, nb);
    float pa[3], pb[3];
    const float pos[3] = {p0.x, p0.y, p0.z};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      pa[r] = pos[r] + (R[r][0] * (na[0] * s[0]) + R[r][1] * (na[1] * s[1]) + R[r][2] * (na[2] * s[2]));
      pb[r] = pos[r] + (R[r][0] * (nb[0] * s[0]) + R[r][1] * (nb[1] * s[1]) + R[r][2] * (nb[2] * s[2]));
    }
    const float ls = logf(f.densify1[2]);
    const float4 scale = make_float4(p1.x - ls, p1.y - ls, p1.z - ls, 1.0f);
    a.P[i] = make_float4(pa[0], pa[1], pa[2], p0.w);
    a.P[a.cap + i] = scale;
    a.P[target] = make_float4(pb[0], pb[1], pb[2], p0.w);
    a.P[a.cap + target] = scale;
    clear_moments(a, i);
  }
  a.P[2u * a.cap + target] = q;
  a.P[3u * a.cap + target] = p3;
}

__global__ void __launch_bounds__(256) k_reset_opacity(float4* P, float4* M, float4* V, uint32_t cap, uint32_t slots,
                                                       float max_logit) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= slots || P[cap + i].w < 0.5f) return;
  P[i].w = fminf(P[i].w, max_logit);
  M[i].w = 0.0f;
  V[i].w = 0.0f;
}

}  // namespace

void launch_pair_sum(const ViewBuffers& vb, uint32_t n_items, const uint32_t* depth_order, const uint32_t* first,
                     const float4* pair_grads, const uint32_t* d_pairs, uint32_t accept, cudaStream_t st) {
  if (n_items == 0u) return;
  PairSumArgs a{n_items, depth_order, first, pair_grads, vb.grad2d, d_pairs, accept};
  const uint32_t per_block = kSumWarps * 32u;
  k_pair_sum<<<(n_items + per_block - 1u) / per_block, per_block, 0, st>>>(a);
}

template <bool MOTION, bool WORD>
void step_degree_word(uint32_t degree, dim3 grid, dim3 block, cudaStream_t st, const StepArgs& a) {
  switch (degree) {
    case 0: k_step_geometry<0, MOTION, WORD><<<grid, block, 0, st>>>(a); break;
    case 1:
      k_step_sh<1, MOTION, WORD><<<grid, block, 0, st>>>(a);
      k_step_geometry<1, MOTION, WORD><<<grid, block, 0, st>>>(a);
      break;
    case 2:
      k_step_sh<2, MOTION, WORD><<<grid, block, 0, st>>>(a);
      k_step_geometry<2, MOTION, WORD><<<grid, block, 0, st>>>(a);
      break;
    default:
      k_step_sh<3, MOTION, WORD><<<grid, block, 0, st>>>(a);
      k_step_geometry<3, MOTION, WORD><<<grid, block, 0, st>>>(a);
      break;
  }
}

// The view word's reads are compiled in or out (WORD), so neither mode branches on it.
template <bool MOTION>
void step_degree(uint32_t degree, dim3 grid, dim3 block, cudaStream_t st, const StepArgs& a) {
  if (a.view_word) step_degree_word<MOTION, true>(degree, grid, block, st, a);
  else step_degree_word<MOTION, false>(degree, grid, block, st, a);
}

StepArgs step_args(const StepPointers& sp, const Model& m, const ViewBuffers& vb, const uint32_t* d_pairs,
                   uint32_t accept, const Motion* motion) {
  return StepArgs{sp.frames, sp.n_views, m.cap,    m.slots,     m.P,     m.M,    m.V,
                  m.SH,      m.MSH,      m.VSH,    m.stats,     vb.splat, vb.tiles, vb.grad2d,
                  vb.dir_grad, vb.view_word, d_pairs, accept, motion ? *motion : Motion{}};
}

void launch_step(const StepPointers& sp, const Model& m, uint32_t degree, const ViewBuffers& vb,
                 const uint32_t* d_pairs, uint32_t accept, const Motion* motion, cudaStream_t st) {
  if (m.slots == 0u) return;
  const StepArgs a = step_args(sp, m, vb, d_pairs, accept, motion);
  const dim3 grid((m.slots + 127u) / 128u), block(128);
  if (motion != nullptr) step_degree<true>(degree, grid, block, st, a);
  else step_degree<false>(degree, grid, block, st, a);
}

uint32_t pose_blocks(uint32_t slots) { return (slots + 127u) / 128u; }

template <bool MOTION>
void pose_degree(uint32_t degree, dim3 grid, dim3 block, cudaStream_t st, const StepArgs& a, float* partial) {
  switch (degree) {
    case 0: k_pose_grad<0, MOTION><<<grid, block, 0, st>>>(a, partial); break;
    case 1: k_pose_grad<1, MOTION><<<grid, block, 0, st>>>(a, partial); break;
    case 2: k_pose_grad<2, MOTION><<<grid, block, 0, st>>>(a, partial); break;
    default: k_pose_grad<3, MOTION><<<grid, block, 0, st>>>(a, partial); break;
  }
}

void launch_pose_grad(const StepPointers& sp, const Model& m, uint32_t degree, const ViewBuffers& vb,
                      const uint32_t* d_pairs, uint32_t accept, const Motion* motion, float* partial, double* out,
                      uint32_t stride, cudaStream_t st) {
  const uint32_t blocks = pose_blocks(m.slots);
  if (blocks > 0u) {
    const StepArgs a = step_args(sp, m, vb, d_pairs, accept, motion);
    const dim3 grid(blocks, sp.n_views), block(128);
    if (motion != nullptr) pose_degree<true>(degree, grid, block, st, a, partial);
    else pose_degree<false>(degree, grid, block, st, a, partial);
  }
  k_pose_reduce<<<sp.n_views, 256, 0, st>>>(sp.frames, partial, blocks, out, stride);
}

uint32_t motion_blocks(uint32_t slots, int sm_count) {
  return std::min((slots + 127u) / 128u, uint32_t(std::max(sm_count, 1)) * 4u);
}

void launch_motion_grad(const StepPointers& sp, const Model& m, uint32_t degree, const ViewBuffers& vb,
                        const uint32_t* d_pairs, uint32_t accept, const Motion& motion, float* partial, double* out,
                        cudaStream_t st) {
  const uint32_t blocks = motion_blocks(m.slots, sp.sm_count);
  if (blocks > 0u) {
    const StepArgs a = step_args(sp, m, vb, d_pairs, accept, &motion);
    const dim3 grid(blocks, sp.n_views), block(128);
    switch (degree) {
      case 0: k_motion_grad<0><<<grid, block, 0, st>>>(a, partial); break;
      case 1: k_motion_grad<1><<<grid, block, 0, st>>>(a, partial); break;
      case 2: k_motion_grad<2><<<grid, block, 0, st>>>(a, partial); break;
      default: k_motion_grad<3><<<grid, block, 0, st>>>(a, partial); break;
    }
  }
  k_motion_reduce<<<dim3(std::max(motion.nodes, 1u), sp.n_views), 64, 0, st>>>(sp.frames, partial, blocks, out);
}

void launch_motion_bind(const Model& m, const Motion& motion, cudaStream_t st) {
  if (m.slots == 0u || motion.nodes == 0u) return;
  k_motion_bind<<<(m.slots + 127u) / 128u, 128, 0, st>>>(m.P, m.cap, m.slots, motion.rest, motion.nodes, motion.bind);
}

void launch_densify(const gs_frame_data* d_frame, const Model& m, const DensifyScratch& ds, const SortScratch& ss,
                    cudaStream_t st, int* launches) {
  if (m.slots == 0u) return;
  DensifyArgs a{d_frame, m.cap, m.slots, m.sh_stride, m.P, m.M, m.V, m.SH, m.MSH, m.VSH, m.stats,
                ds.spawn, ds.release, ds.wants, ds.free_pos, ds.spawn_pos, ds.free_list, ds.counters};
  const uint32_t blocks = (m.slots + 127u) / 128u;
  cudaMemsetAsync(ds.counters, 0, 4 * sizeof(uint32_t), st);
  k_densify_mark<<<blocks, 128, 0, st>>>(a);
  exclusive_scan(ss, ds.release, nullptr, ds.free_pos, m.slots, ds.counters + 0, st, launches);
  exclusive_scan(ss, ds.wants, nullptr, ds.spawn_pos, m.slots, ds.counters + 1, st, launches);
  k_free_list<<<blocks, 128, 0, st>>>(a);
  k_densify_spawn<<<blocks, 128, 0, st>>>(a, m.cap);
  cudaMemsetAsync(m.stats, 0, sizeof(float4) * m.cap, st);
  if (launches) *launches += 3;
}

void launch_reset_opacity(const Model& m, float max_logit, cudaStream_t st) {
  if (m.slots == 0u) return;
  k_reset_opacity<<<(m.slots + 255u) / 256u, 256, 0, st>>>(m.P, m.M, m.V, m.cap, m.slots, max_logit);
}

}  // namespace gsk
