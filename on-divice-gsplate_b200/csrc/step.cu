// Optimizer side of the step: per-gaussian pair sums (train_pair_sum.comp:17-32), the
// projection backward fused with Adam on all parameters (train_step.glsl:62-240 and
// train_step_sh.comp:21-44), adaptive density control (train_densify_mark.comp,
// train_densify_spawn.comp) and the opacity reset (train_reset_opacity.comp).
//
// k_step reads each slot's parameters, SH and moments once, back-propagates every view's
// summed 2D gradient through that view's projection (views of one step add up), and
// takes one Adam step on the 16 parameters and the active SH coefficients. HBM-bound:
// params, SH and both moment sets are read and written once per step.
#include "gs_kernels.h"

namespace gsk {
namespace {

struct PairSumArgs {
  uint32_t n_views, cap, slots;
  const uint32_t* tiles;
  const uint32_t* offsets;
  const float4* pair_grads;
  float4* grad2d;
  const uint32_t* d_pairs;
  uint32_t accept;
};

__global__ void __launch_bounds__(128) k_pair_sum(PairSumArgs a) {
  if (*a.d_pairs > a.accept) return;
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.n_views * a.slots) return;
  const uint32_t v = idx / a.slots, i = idx - v * a.slots;
  const size_t g = size_t(v) * a.cap + i;
  const uint32_t count = a.tiles[g];
  float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f), s1 = s0, s2 = s0;
  if (count > 0u) {
    const size_t first = a.offsets[g];
    for (uint32_t k = 0; k < count; ++k) {
      const float4 x = a.pair_grads[(first + k) * 3u], y = a.pair_grads[(first + k) * 3u + 1u],
                   z = a.pair_grads[(first + k) * 3u + 2u];
      s0.x += x.x; s0.y += x.y; s0.z += x.z; s0.w += x.w;
      s1.x += y.x; s1.y += y.y; s1.z += y.z; s1.w += y.w;
      s2.x += z.x; s2.y += z.y; s2.z += z.z; s2.w += z.w;
    }
  }
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
  const uint32_t* d_pairs;
  uint32_t accept;
};

__device__ __forceinline__ float adam1(float p, float g, float& m, float& v, float lr, float b1, float b2, float c1,
                                       float c2, float eps) {
  m = g * (1.0f - b1) + m * b1;
  v = g * g * (1.0f - b2) + v * b2;
  return p - lr * (m * c1) / (sqrtf(v * c2) + eps);
}

template <int DEG>
__global__ void __launch_bounds__(128) k_step(StepArgs a) {
  __shared__ gs_frame_data s_frames[kMaxViews];
  {
    const uint32_t words = a.n_views * uint32_t(sizeof(gs_frame_data) / 4);
    for (uint32_t k = threadIdx.x; k < words; k += blockDim.x)
      reinterpret_cast<uint32_t*>(s_frames)[k] = reinterpret_cast<const uint32_t*>(a.frames)[k];
  }
  __syncthreads();
  // More pairs than the buffers hold: gradients are incomplete, leave everything as it
  // was (train_step.glsl:247-251); the host grows the buffers and runs the step again.
  if (*a.d_pairs > a.accept) return;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.slots) return;
  constexpr int K = DEG == 0 ? 0 : (DEG + 1) * (DEG + 1) - 1;
  float4 p0 = a.P[i], p1 = a.P[a.cap + i], q = a.P[2u * a.cap + i], p3 = a.P[3u * a.cap + i];
  if (p1.w < 0.5f) return;  // free slot

  float g16[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) g16[k] = 0.0f;
  float gsh[K > 0 ? 3 * K : 1];
#pragma unroll
  for (int k = 0; k < 3 * K; ++k) gsh[k] = 0.0f;
  uint32_t drew = 0u;

  // View-independent: normalised quaternion, R, scales, M = R S, Sigma = M M^T.
  const float qlen = fmaxf(sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w), 1e-12f);
  const float qn[4] = {q.x / qlen, q.y / qlen, q.z / qlen, q.w / qlen};
  float R[3][3];
  quat_to_matrix(qn[0], qn[1], qn[2], qn[3], R);
  const float s[3] = {expf(p1.x), expf(p1.y), expf(p1.z)};
  float Mm[3][3], Sig[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) Mm[r][c] = R[r][c] * s[c];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) Sig[r][c] = Mm[r][0] * Mm[c][0] + Mm[r][1] * Mm[c][1] + Mm[r][2] * Mm[c][2];
  const float opacity = sigmoidf(p0.w);
  float4 st = a.stats[i];
  bool seen = false;

  for (uint32_t v = 0; v < a.n_views; ++v) {
    const size_t g = size_t(v) * a.cap + i;
    if (a.tiles[g] == 0u) continue;
    seen = true;
    const gs_frame_data& f = s_frames[v];
    const float4 a0 = a.grad2d[g * 3u], a1 = a.grad2d[g * 3u + 1u], a2 = a.grad2d[g * 3u + 2u];
    if (a0.x != 0.f || a0.y != 0.f || a0.z != 0.f || a0.w != 0.f || a1.x != 0.f || a1.y != 0.f || a1.z != 0.f ||
        a1.w != 0.f || a2.x != 0.f || a2.y != 0.f || a2.z != 0.f || a2.w != 0.f)
      drew |= 1u;
    const float dmx = a0.x, dmy = a0.y;
    const float ga = a0.z, gb = a0.w, gc = a1.x;
    const float dop = a1.y;
    float dcol[3] = {a1.z, a1.w, a2.x};
    const float width = float(f.image[0]), height = float(f.image[1]);
    const float nx = 0.5f * width, ny = 0.5f * height;
    // Densification statistics: the view-space positional gradient in NDC units.
    st.x += sqrtf((dmx * nx) * (dmx * nx) + (dmy * ny) * (dmy * ny));
    st.y += 1.0f;
    st.z = fmaxf(st.z, a.splat[g * 3u + 1u].w);
    st.w += sqrtf((a2.y * nx) * (a2.y * nx) + (a2.z * ny) * (a2.z * ny));

    // Recompute the projection.
    float t[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) t[r] = f.rot[r][0] * p0.x + f.rot[r][1] * p0.y + f.rot[r][2] * p0.z + f.rot[r][3];
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
      T[0][c] = j00 * f.rot[0][c] + j02 * f.rot[2][c];
      T[1][c] = j11 * f.rot[1][c] + j12 * f.rot[2][c];
    }
    float TS[2][3];  // T Sigma
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) TS[r][c] = T[r][0] * Sig[0][c] + T[r][1] * Sig[1][c] + T[r][2] * Sig[2][c];
    const float A = TS[0][0] * T[0][0] + TS[0][1] * T[0][1] + TS[0][2] * T[0][2] + kDilation;
    const float B = TS[1][0] * T[0][0] + TS[1][1] * T[0][1] + TS[1][2] * T[0][2];
    const float C = TS[1][0] * T[1][0] + TS[1][1] * T[1][1] + TS[1][2] * T[1][2] + kDilation;
    const float D = A * C - B * B;

    // Colour -> SH coefficients and view direction.
    float dr[3] = {p0.x - f.cam_pos[0], p0.y - f.cam_pos[1], p0.z - f.cam_pos[2]};
    const float dir_len = fmaxf(sqrtf(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]), 1e-12f);
    const float dir[3] = {dr[0] / dir_len, dr[1] / dir_len, dr[2] / dir_len};
    const uint32_t clamped = __float_as_uint(a.splat[g * 3u + 2u].w);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if (clamped & (1u << c)) dcol[c] = 0.0f;
    if (dcol[0] != 0.0f || dcol[1] != 0.0f || dcol[2] != 0.0f) drew |= 2u;
    float basis[16];
    sh_basis<DEG>(dir[0], dir[1], dir[2], basis);
#pragma unroll
    for (int c = 0; c < 3; ++c) g16[12 + c] += basis[0] * dcol[c];
    float ddir[3] = {0.f, 0.f, 0.f};
    if constexpr (K > 0) {
      float db[16][3];
      sh_basis_grad<DEG>(dir[0], dir[1], dir[2], db);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const float w = a.SH[size_t(3 * k) * a.cap + i] * dcol[0] + a.SH[size_t(3 * k + 1) * a.cap + i] * dcol[1] +
                        a.SH[size_t(3 * k + 2) * a.cap + i] * dcol[2];
        ddir[0] += w * db[k + 1][0];
        ddir[1] += w * db[k + 1][1];
        ddir[2] += w * db[k + 1][2];
        gsh[3 * k] += basis[k + 1] * dcol[0];
        gsh[3 * k + 1] += basis[k + 1] * dcol[1];
        gsh[3 * k + 2] += basis[k + 1] * dcol[2];
      }
    }
    const float dd = dir[0] * ddir[0] + dir[1] * ddir[1] + dir[2] * ddir[2];
    float ddir_raw[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) ddir_raw[c] = (ddir[c] - dir[c] * dd) / dir_len;

    g16[3] += dop * opacity * (1.0f - opacity);

    // Conic -> dilated 2D covariance.
    const float inv_d2 = 1.0f / (D * D);
    const float gA = (-C * C * ga + B * C * gb - B * B * gc) * inv_d2;
    const float gB = (2.0f * B * C * ga - (D + 2.0f * B * B) * gb + 2.0f * A * B * gc) * inv_d2;
    const float gC = (-B * B * ga + A * B * gb - A * A * gc) * inv_d2;
    const float G2[2][2] = {{gA, 0.5f * gB}, {0.5f * gB, gC}};
    // dSigma = T^T G2 T, dT = 2 G2 T Sigma, dJ = dT W^T (rows 0, 1; row 2 of J is zero).
    float G2T[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) G2T[r][c] = G2[r][0] * T[0][c] + G2[r][1] * T[1][c];
    float dSig[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) dSig[r][c] = T[0][r] * G2T[0][c] + T[1][r] * G2T[1][c];
    float dT[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        dT[r][c] = 2.0f * (G2[r][0] * TS[0][c] + G2[r][1] * TS[1][c]);
    float dJ[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) dJ[r][c] = dT[r][0] * f.rot[c][0] + dT[r][1] * f.rot[c][1] + dT[r][2] * f.rot[c][2];
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
#pragma unroll
    for (int c = 0; c < 3; ++c) g16[c] += f.rot[0][c] * dt[0] + f.rot[1][c] * dt[1] + f.rot[2][c] * dt[2] + ddir_raw[c];

    // 3D covariance -> log scale and rotation.
    float dM[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) dM[r][c] = 2.0f * (dSig[r][0] * Mm[0][c] + dSig[r][1] * Mm[1][c] + dSig[r][2] * Mm[2][c]);
#pragma unroll
    for (int c = 0; c < 3; ++c) g16[4 + c] += (dM[0][c] * R[0][c] + dM[1][c] * R[1][c] + dM[2][c] * R[2][c]) * s[c];
    float gR[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) gR[r][c] = dM[r][c] * s[c];
    const float w = qn[0], x = qn[1], y = qn[2], z = qn[3];
    float dq[4];
    dq[0] = 2.0f * (-z * gR[0][1] + y * gR[0][2] + z * gR[1][0] - x * gR[1][2] - y * gR[2][0] + x * gR[2][1]);
    dq[1] = 2.0f * (y * gR[0][1] + z * gR[0][2] + y * gR[1][0] - 2.0f * x * gR[1][1] - w * gR[1][2] + z * gR[2][0] +
                    w * gR[2][1] - 2.0f * x * gR[2][2]);
    dq[2] = 2.0f * (-2.0f * y * gR[0][0] + x * gR[0][1] + w * gR[0][2] + x * gR[1][0] + z * gR[1][2] - w * gR[2][0] +
                    z * gR[2][1] - 2.0f * y * gR[2][2]);
    dq[3] = 2.0f * (-2.0f * z * gR[0][0] - w * gR[0][1] + x * gR[0][2] + w * gR[1][0] - 2.0f * z * gR[1][1] +
                    y * gR[1][2] + x * gR[2][0] + y * gR[2][1]);
    const float qd = qn[0] * dq[0] + qn[1] * dq[1] + qn[2] * dq[2] + qn[3] * dq[3];
#pragma unroll
    for (int k = 0; k < 4; ++k) g16[8 + k] += (dq[k] - qn[k] * qd) / qlen;
  }
  if (seen) a.stats[i] = st;

  // Adam with the step's constants (the first view's frame).
  const gs_frame_data& f0 = s_frames[0];
  const bool sparse = (f0.model[3] & GS_FLAG_SPARSE_ADAM) != 0u;
  const float b1 = f0.adam[0], b2 = f0.adam[1], eps = f0.adam[2], c1 = f0.bias[0], c2 = f0.bias[1];
  if (!sparse || (drew & 1u)) {
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
  if constexpr (K > 0) {
    // train_step_sh.comp:34-35: with sparse Adam, a zero colour gradient keeps the SH.
    if (!sparse || (drew & 2u)) {
      const float lr = f0.lr1[1];
#pragma unroll
      for (int k = 0; k < 3 * K; ++k) {
        const size_t o = size_t(k) * a.cap + i;
        float m = a.MSH[o], v = a.VSH[o];
        a.SH[o] = adam1(a.SH[o], gsh[k], m, v, lr, b1, b2, c1, c2, eps);
        a.MSH[o] = m;
        a.VSH[o] = v;
      }
    }
  }
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

void launch_pair_sum(const StepPointers& sp, const ViewBuffers& vb, uint32_t cap, uint32_t slots,
                     const float4* pair_grads, const uint32_t* d_pairs, uint32_t accept, cudaStream_t st) {
  const uint32_t n = sp.n_views * slots;
  if (n == 0u) return;
  PairSumArgs a{sp.n_views, cap, slots, vb.tiles, vb.offsets, pair_grads, vb.grad2d, d_pairs, accept};
  k_pair_sum<<<(n + 127u) / 128u, 128, 0, st>>>(a);
}

void launch_step(const StepPointers& sp, const Model& m, uint32_t degree, const ViewBuffers& vb,
                 const uint32_t* d_pairs, uint32_t accept, cudaStream_t st) {
  if (m.slots == 0u) return;
  StepArgs a{sp.frames, sp.n_views, m.cap, m.slots, m.P, m.M, m.V, m.SH, m.MSH, m.VSH, m.stats,
             vb.splat, vb.tiles, vb.grad2d, d_pairs, accept};
  const dim3 grid((m.slots + 127u) / 128u), block(128);
  switch (degree) {
    case 0: k_step<0><<<grid, block, 0, st>>>(a); break;
    case 1: k_step<1><<<grid, block, 0, st>>>(a); break;
    case 2: k_step<2><<<grid, block, 0, st>>>(a); break;
    default: k_step<3><<<grid, block, 0, st>>>(a); break;
  }
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
