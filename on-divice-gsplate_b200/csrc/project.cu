// Projection: EWA 2D covariance, SH colour, opacity-aware tile count and the 16-bit
// depth key of every slot, for every view of the step (train_project.comp:26-112).
//
// One thread per (view, slot). A block projects 128 consecutive slots into one view, and
// the views of a slot chunk are neighbouring blocks, so a chunk's parameters (four
// coalesced float4 planes, the SH planes when visible) come from HBM once per step and
// from L2 for the other views. HBM-bound: per slot and view it writes 48 B of splat
// record, 16 B of footprint, a tile count and a depth key/value pair, and for slots with
// pairs the tile-row spans the count walked, packed for the pair emission (which then
// reads 16 B instead of repeating the walk's divisions and square roots). Capped at 72
// registers, 7 blocks per SM. A thread per slot looping over the views (128 registers,
// 4 blocks per SM) measured 0.54 ms against 0.43 ms for 8 views of 1M slots (0.48 ms with
// the spans, which take 0.09 ms off the emission).
//
// With MOTION (any view of the step has GS_FLAG_MOTION) a slot is first moved with the
// subject in the views that have the flag (train_project.comp:36-41): its position by the
// node blend, its covariance by the blended turn U (world -> camera becomes V U for it),
// and the SH colour is looked up in its own rest frame (direction U^T (x - camera)).
#include "gs_kernels.h"
#include "motion.cuh"

namespace gsk {
namespace {

struct ProjectArgs {
  const gs_frame_data* frames;
  uint32_t n_views, slots, cap;
  const float4* P;
  const float* SH;
  float4* splat;
  float4* foot;
  uint4* spans;
  uint32_t* tiles;
  uint32_t* dkeys;
  uint32_t* dvals;
  float4* grad2d;  // zeroed when non-null (atomic backward), the view word in its 12th float
  Motion motion;
};

template <int DEG, bool MOTION>
__global__ void __launch_bounds__(128, 7) k_project(ProjectArgs a) {
  // Block b projects 128 slots into one view: view b % n_views of slot chunk b / n_views,
  // so the views of a chunk run in neighbouring blocks and re-read its parameters from L2.
  __shared__ gs_frame_data s_frame;
  const uint32_t v = blockIdx.x % a.n_views, chunk = blockIdx.x / a.n_views;
  {
    constexpr uint32_t words = uint32_t(sizeof(gs_frame_data) / 4);
    for (uint32_t k = threadIdx.x; k < words; k += blockDim.x)
      reinterpret_cast<uint32_t*>(&s_frame)[k] = reinterpret_cast<const uint32_t*>(a.frames + v)[k];
  }
  __syncthreads();
  const uint32_t i = chunk * blockDim.x + threadIdx.x;
  if (i >= a.slots) return;
  constexpr int kCoeffs = DEG == 0 ? 0 : (DEG + 1) * (DEG + 1) - 1;

  const float4 p0 = a.P[i], p1 = a.P[a.cap + i], q = a.P[2u * a.cap + i], p3 = a.P[3u * a.cap + i];
  const float opacity = sigmoidf(p0.w);
  const bool alive = p1.w > 0.5f && opacity >= kMinAlpha;

  // View-independent part: Sigma = R S S^T R^T.
  float Sig[3][3];
  {
    const float qlen = fmaxf(sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w), 1e-12f);
    float R[3][3];
    quat_to_matrix(q.x / qlen, q.y / qlen, q.z / qlen, q.w / qlen, R);
    const float s[3] = {expf(p1.x), expf(p1.y), expf(p1.z)};
    float M[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) M[r][c] = R[r][c] * s[c];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) Sig[r][c] = M[r][0] * M[c][0] + M[r][1] * M[c][1] + M[r][2] * M[c][2];
  }
  {
    const gs_frame_data& f = s_frame;
    const size_t g = size_t(v) * a.cap + i;
    float4 o0 = make_float4(0.f, 0.f, 0.f, 0.f), o1 = o0, o2 = o0, o3 = o0;
    uint32_t tiles = 0u;
    uint4 spans = make_uint4(0u, 0u, 0u, 0u);
    float x0 = p0.x, x1 = p0.y, x2 = p0.z;
    float W[3][3];  // rest frame -> camera, for the covariance
    float U[3][3];  // the orientation's turn (MOTION only)
    bool moved = false;
    if constexpr (MOTION) {
      if ((f.model[3] & GS_FLAG_MOTION) != 0u && p1.w > 0.5f) {
        Deformed d;
        deform(a.motion, a.motion.views + size_t(v) * kMaxMotionNodes, i, p0.x, p0.y, p0.z, d);
        x0 = d.x[0];
        x1 = d.x[1];
        x2 = d.x[2];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) U[r][c] = d.U[r][c];
        moved = true;
      }
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        W[r][c] = moved ? f.rot[r][0] * U[0][c] + f.rot[r][1] * U[1][c] + f.rot[r][2] * U[2][c] : f.rot[r][c];
    const float tz = f.rot[2][0] * x0 + f.rot[2][1] * x1 + f.rot[2][2] * x2 + f.rot[2][3];
    if (alive && tz > kNear) {
      const float tx3 = f.rot[0][0] * x0 + f.rot[0][1] * x1 + f.rot[0][2] * x2 + f.rot[0][3];
      const float ty3 = f.rot[1][0] * x0 + f.rot[1][1] * x1 + f.rot[1][2] * x2 + f.rot[1][3];
      const float fx = f.intrinsics[0], fy = f.intrinsics[1], cx = f.intrinsics[2], cy = f.intrinsics[3];
      const float width = float(f.image[0]), height = float(f.image[1]);
      const float inv_z = 1.0f / tz;
      const float mx = fx * tx3 * inv_z + cx, my = fy * ty3 * inv_z + cy;
      const float lim_x = 1.3f * fmaxf(cx, width - cx) / fx;
      const float lim_y = 1.3f * fmaxf(cy, height - cy) / fy;
      const float tx = clampf(tx3 * inv_z, -lim_x, lim_x);
      const float ty = clampf(ty3 * inv_z, -lim_y, lim_y);
      const float j00 = fx * inv_z, j02 = -fx * tx * inv_z, j11 = fy * inv_z, j12 = -fy * ty * inv_z;
      float T0[3], T1[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T0[c] = j00 * W[0][c] + j02 * W[2][c];
        T1[c] = j11 * W[1][c] + j12 * W[2][c];
      }
      float u0[3], u1[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        u0[k] = T0[0] * Sig[0][k] + T0[1] * Sig[1][k] + T0[2] * Sig[2][k];
        u1[k] = T1[0] * Sig[0][k] + T1[1] * Sig[1][k] + T1[2] * Sig[2][k];
      }
      const float ca = u0[0] * T0[0] + u0[1] * T0[1] + u0[2] * T0[2] + kDilation;
      const float cb = u1[0] * T0[0] + u1[1] * T0[1] + u1[2] * T0[2];
      const float cc = u1[0] * T1[0] + u1[1] * T1[1] + u1[2] * T1[2] + kDilation;
      const float det = ca * cc - cb * cb;
      if (det > 0.0f) {
        const float mid = 0.5f * (ca + cc);
        const float lambda = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
        const float sigma = sqrtf(lambda);
        const float thr = footprint_threshold(opacity);
        tiles = footprint_count_spans(mx, my, ca, cb, cc, thr, f.image[0], f.image[1], spans);
        if (tiles > 0u) {
          o3 = make_float4(ca, cb, cc, thr);
          float dx = x0 - f.cam_pos[0], dy = x1 - f.cam_pos[1], dz = x2 - f.cam_pos[2];
          if (moved) {  // into the rest frame: U^T (x - camera)
            const float rx = U[0][0] * dx + U[1][0] * dy + U[2][0] * dz;
            const float ry = U[0][1] * dx + U[1][1] * dy + U[2][1] * dz;
            const float rz = U[0][2] * dx + U[1][2] * dy + U[2][2] * dz;
            dx = rx;
            dy = ry;
            dz = rz;
          }
          const float dl = sqrtf(dx * dx + dy * dy + dz * dz);
          dx /= dl;
          dy /= dl;
          dz /= dl;
          float basis[16];
          sh_basis<DEG>(dx, dy, dz, basis);
          float col[3] = {basis[0] * p3.x, basis[0] * p3.y, basis[0] * p3.z};
          if constexpr (kCoeffs > 0) {
#pragma unroll
            for (int k = 0; k < kCoeffs; ++k) {
              col[0] += basis[k + 1] * a.SH[size_t(3 * k) * a.cap + i];
              col[1] += basis[k + 1] * a.SH[size_t(3 * k + 1) * a.cap + i];
              col[2] += basis[k + 1] * a.SH[size_t(3 * k + 2) * a.cap + i];
            }
          }
          uint32_t clamped = 0u;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            col[c] += 0.5f;
            if (col[c] < 0.0f) clamped |= 1u << c;
            col[c] = fmaxf(col[c], 0.0f);
          }
          const float inv_det = 1.0f / det;
          o0 = make_float4(mx, my, tz, opacity);
          o1 = make_float4(cc * inv_det, -cb * inv_det, ca * inv_det, ceilf(3.0f * sigma));
          o2 = make_float4(col[0], col[1], col[2], __uint_as_float(clamped));
        }
      }
    }
    a.splat[g * 3u] = o0;
    a.splat[g * 3u + 1u] = o1;
    a.splat[g * 3u + 2u] = o2;
    a.foot[g] = o3;
    if (tiles > 0u) a.spans[g] = spans;  // emission reads it only for slots with pairs
    a.tiles[g] = tiles;
    const uint32_t key =
        tiles > 0u ? uint32_t(clampf(log2f(o0.z / kNear) / kLogRange, 0.0f, 1.0f) * 65535.0f) : 0xffffu;
    const size_t e = size_t(v) * a.slots + i;
    a.dkeys[e] = (v << 16) | key;
    a.dvals[e] = uint32_t(g);
    if (a.grad2d != nullptr) {  // zeroed for the backward's atomics, with the view word
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      a.grad2d[g * 3u] = z;
      a.grad2d[g * 3u + 1u] = z;
      const float word = tiles > 0u ? pack_view_word(o1.w, __float_as_uint(o2.w)) : 0.f;
      a.grad2d[g * 3u + 2u] = make_float4(0.f, 0.f, 0.f, word);
    }
  }
}

}  // namespace

template <bool MOTION>
void project_degree(uint32_t degree, dim3 grid, dim3 block, cudaStream_t st, const ProjectArgs& a) {
  switch (degree) {
    case 0: k_project<0, MOTION><<<grid, block, 0, st>>>(a); break;
    case 1: k_project<1, MOTION><<<grid, block, 0, st>>>(a); break;
    case 2: k_project<2, MOTION><<<grid, block, 0, st>>>(a); break;
    default: k_project<3, MOTION><<<grid, block, 0, st>>>(a); break;
  }
}

void launch_project(const StepPointers& sp, const Model& m, uint32_t degree, const ViewBuffers& vb,
                    uint32_t* depth_keys, uint32_t* depth_vals, bool zero_grad2d, const Motion* motion,
                    cudaStream_t st) {
  if (m.slots == 0 || sp.n_views == 0) return;
  ProjectArgs a{sp.frames, sp.n_views, m.slots, m.cap, m.P, m.SH, vb.splat, vb.foot, vb.spans, vb.tiles,
                depth_keys, depth_vals, zero_grad2d ? vb.grad2d : nullptr, motion ? *motion : Motion{}};
  const dim3 grid(((m.slots + 127u) / 128u) * sp.n_views), block(128);
  if (motion != nullptr) project_degree<true>(degree, grid, block, st, a);
  else project_degree<false>(degree, grid, block, st, a);
}

}  // namespace gsk
