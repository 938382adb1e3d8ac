// Device-side definitions shared by the training-step kernels (sm_100a).
//
// Constants, FrameData access and the footprint arithmetic of
// engine/shaders/train_common.glsl. The footprint helpers use explicit
// round-to-nearest intrinsics (no FMA contraction): the reference marks them
// `precise` so that train_project's tile count and train_emit's tile walk agree
// to the bit (train_common.glsl:163-168); here they also agree to the bit with
// a CPU evaluation of the same expressions.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gs_cuda.h"

namespace gsk {

constexpr uint32_t kTile = 16;
constexpr uint32_t kTilePixels = kTile * kTile;
constexpr float kNear = 0.02f;
constexpr float kLogRange = 15.6096404744f;  // log2(kFar / kNear), kFar = 1000 (train_common.glsl:65-66)
constexpr float kDilation = 0.3f;
constexpr float kMinAlpha = 1.0f / 255.0f;
constexpr float kMaxAlpha = 0.99f;
constexpr float kMinTransmittance = 1e-4f;
constexpr uint32_t kMaxViews = GS_MAX_VIEWS;

// Views of one step, laid out for the flattened (view, tile) and (view, pixel) spaces.
// Lives in device memory (uploaded with the views' FrameData each step), so the step's
// launches do not change when the views do and the step can be replayed as a CUDA graph.
struct ViewTable {
  uint32_t n_views;
  uint32_t total_tiles;
  uint32_t total_pixels;
  uint32_t pad;
  uint32_t tile_base[kMaxViews + 1];   // global tile index of each view's tile 0
  uint32_t pixel_base[kMaxViews + 1];  // global pixel index of each view's pixel 0
  const uint32_t* target[kMaxViews];   // each view's RGBA8 target (width x height), or null
};

// What one step uploads: the view table and each view's FrameData.
struct StepTable {
  ViewTable vt;
  gs_frame_data frames[kMaxViews];
};

__device__ __forceinline__ uint32_t view_of_tile(const ViewTable* vt, uint32_t gtile) {
  const uint32_t n = vt->n_views;
  uint32_t v = 0;
  while (v + 1 < n && gtile >= vt->tile_base[v + 1]) ++v;
  return v;
}

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }
__device__ __forceinline__ float sigmoidf(float x) { return 1.0f / (1.0f + expf(-x)); }

// train_common.glsl:72-78, R[row][col].
__device__ __forceinline__ void quat_to_matrix(float w, float x, float y, float z, float R[3][3]) {
  R[0][0] = 1.0f - 2.0f * (y * y + z * z);
  R[1][0] = 2.0f * (x * y + w * z);
  R[2][0] = 2.0f * (x * z - w * y);
  R[0][1] = 2.0f * (x * y - w * z);
  R[1][1] = 1.0f - 2.0f * (x * x + z * z);
  R[2][1] = 2.0f * (y * z + w * x);
  R[0][2] = 2.0f * (x * z + w * y);
  R[1][2] = 2.0f * (y * z - w * x);
  R[2][2] = 1.0f - 2.0f * (x * x + y * y);
}

__host__ __device__ __forceinline__ int sh_rest_coeffs(uint32_t degree) {
  return degree == 0u ? 0 : int((degree + 1u) * (degree + 1u)) - 1;
}

// Real SH basis up to degree DEG (train_common.glsl:84-109).
template <int DEG>
__device__ __forceinline__ void sh_basis(float x, float y, float z, float b[16]) {
  b[0] = 0.28209479177387814f;
  if (DEG >= 1) {
    b[1] = -0.4886025119029199f * y;
    b[2] = 0.4886025119029199f * z;
    b[3] = -0.4886025119029199f * x;
  }
  if (DEG >= 2) {
    const float xx = x * x, yy = y * y, zz = z * z;
    b[4] = 1.0925484305920792f * x * y;
    b[5] = -1.0925484305920792f * y * z;
    b[6] = 0.31539156525252005f * (2.0f * zz - xx - yy);
    b[7] = -1.0925484305920792f * x * z;
    b[8] = 0.5462742152960396f * (xx - yy);
    if (DEG >= 3) {
      b[9] = -0.5900435899266435f * y * (3.0f * xx - yy);
      b[10] = 2.890611442640554f * x * y * z;
      b[11] = -0.4570457994644658f * y * (4.0f * zz - xx - yy);
      b[12] = 0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
      b[13] = -0.4570457994644658f * x * (4.0f * zz - xx - yy);
      b[14] = 1.445305721320277f * z * (xx - yy);
      b[15] = -0.5900435899266435f * x * (xx - 3.0f * yy);
    }
  }
}

// Derivatives of the basis w.r.t. the unit direction (train_common.glsl:111-140): g[k][axis].
template <int DEG>
__device__ __forceinline__ void sh_basis_grad(float x, float y, float z, float g[16][3]) {
#pragma unroll
  for (int k = 0; k < 16; ++k) g[k][0] = g[k][1] = g[k][2] = 0.0f;
  if (DEG >= 1) {
    const float C1 = 0.4886025119029199f;
    g[1][1] = -C1;
    g[2][2] = C1;
    g[3][0] = -C1;
  }
  if (DEG >= 2) {
    const float xx = x * x, yy = y * y, zz = z * z;
    const float A = 1.0925484305920792f, B = 0.31539156525252005f, C = 0.5462742152960396f;
    g[4][0] = A * y; g[4][1] = A * x;
    g[5][1] = -A * z; g[5][2] = -A * y;
    g[6][0] = B * (-2.0f * x); g[6][1] = B * (-2.0f * y); g[6][2] = B * (4.0f * z);
    g[7][0] = -A * z; g[7][2] = -A * x;
    g[8][0] = C * (2.0f * x); g[8][1] = C * (-2.0f * y);
    if (DEG >= 3) {
      const float D = -0.5900435899266435f, E = 2.890611442640554f, F = -0.4570457994644658f;
      const float G = 0.3731763325901154f, H = 1.445305721320277f;
      g[9][0] = D * (6.0f * x * y); g[9][1] = D * (3.0f * xx - 3.0f * yy);
      g[10][0] = E * (y * z); g[10][1] = E * (x * z); g[10][2] = E * (x * y);
      g[11][0] = F * (-2.0f * x * y); g[11][1] = F * (4.0f * zz - xx - 3.0f * yy); g[11][2] = F * (8.0f * y * z);
      g[12][0] = G * (-6.0f * x * z); g[12][1] = G * (-6.0f * y * z); g[12][2] = G * (6.0f * zz - 3.0f * xx - 3.0f * yy);
      g[13][0] = F * (4.0f * zz - 3.0f * xx - yy); g[13][1] = F * (-2.0f * x * y); g[13][2] = F * (8.0f * x * z);
      g[14][0] = H * (2.0f * x * z); g[14][1] = H * (-2.0f * y * z); g[14][2] = H * (xx - yy);
      g[15][0] = D * (3.0f * xx - 3.0f * yy); g[15][1] = D * (-6.0f * x * y);
    }
  }
}

// ---- footprint (train_common.glsl:163-213), round-to-nearest, no contraction ----

__device__ __forceinline__ float footprint_threshold(float opacity) {
  const float t = __fmul_rn(2.0f, logf(__fmul_rn(opacity, 255.0f)));
  return __fadd_rn(__fmul_rn(t, 1.0001f), 1e-4f);
}

__device__ __forceinline__ int2 footprint_pixels(float lo, float hi, uint32_t size) {
  const int n = int(size);
  const int first = clampi(int(clampf(ceilf(lo), -1.0f, float(n))), 0, n);
  const int last = clampi(int(clampf(floorf(hi), -1.0f, float(n))), -1, n - 1);
  return make_int2(first, last);
}

__device__ __forceinline__ int2 footprint_rows(float mx, float my, float cov_c, float t, uint32_t height) {
  const float ey = __fsqrt_rn(__fmul_rn(t, cov_c));
  const float v = __fsub_rn(my, 0.5f);
  return footprint_pixels(__fsub_rn(v, ey), __fadd_rn(v, ey), height);
}

// Tiles [x, y) of tile row ty the ellipse reaches within pixel rows `rows`.
__device__ __forceinline__ uint2 footprint_row_tiles(float mx, float my, float a, float b, float c, float t,
                                                     int2 rows, uint32_t ty, uint32_t width) {
  const float u = __fsub_rn(mx, 0.5f), v = __fsub_rn(my, 0.5f);
  const int r0 = max(int(ty * kTile), rows.x);
  const int r1 = min(int(ty * kTile + kTile - 1u), rows.y);
  const float y0 = __fsub_rn(float(r0), v);
  const float y1 = __fsub_rn(float(r1), v);
  const float k = __fdiv_rn(b, c);
  const float w = __fdiv_rn(__fsub_rn(__fmul_rn(a, c), __fmul_rn(b, b)), c);
  const float side = __fmul_rn(b, __fsqrt_rn(__fdiv_rn(t, a)));
  const float dr = clampf(side, y0, y1);
  const float dl = clampf(-side, y0, y1);
  const float x_max =
      __fadd_rn(__fmul_rn(k, dr), __fsqrt_rn(fmaxf(__fmul_rn(w, __fsub_rn(t, __fdiv_rn(__fmul_rn(dr, dr), c))), 0.0f)));
  const float x_min =
      __fsub_rn(__fmul_rn(k, dl), __fsqrt_rn(fmaxf(__fmul_rn(w, __fsub_rn(t, __fdiv_rn(__fmul_rn(dl, dl), c))), 0.0f)));
  const int2 cols = footprint_pixels(__fadd_rn(u, x_min), __fadd_rn(u, x_max), width);
  if (cols.x > cols.y) return make_uint2(0u, 0u);
  return make_uint2(uint32_t(cols.x) / kTile, uint32_t(cols.y) / kTile + 1u);
}

// The view word of a drawn (view, slot) in fast mode: the footprint radius (an
// integer-valued float; saturated at 2^29 - 1 pixels, far above any pruning threshold)
// above the three clamped-colour bits. Integers below 2^29 convert both ways exactly.
__device__ __forceinline__ float pack_view_word(float radius, uint32_t clamped) {
  const uint32_t r = radius >= 536870911.0f ? 536870911u : uint32_t(radius);
  return __uint_as_float(r << 3 | (clamped & 7u));
}
__device__ __forceinline__ uint32_t view_word_clamped(float w) { return __float_as_uint(w) & 7u; }
__device__ __forceinline__ float view_word_radius(float w) { return float(__float_as_uint(w) >> 3); }

// Tile count of the ellipse, and its tile-row spans packed for the pair emission:
// x = first tile row | rows << 16 | bit 31 when the spans below are complete; y, z, w hold
// rows 0-5 as 16 bits each, first tile (10 bits) | tiles in the row (6 bits) << 10. More
// than 6 rows, a first tile past 1023 or a row of 64 tiles or more leave bit 31 clear (the
// emission walks the rows again).
__device__ __forceinline__ uint32_t footprint_count_spans(float mx, float my, float a, float b, float c, float t,
                                                          uint32_t width, uint32_t height, uint4& packed) {
  const int2 rows = footprint_rows(mx, my, c, t, height);
  uint32_t tiles = 0u;
  packed = make_uint4(0u, 0u, 0u, 0u);
  if (rows.x <= rows.y) {
    const uint32_t ty0 = uint32_t(rows.x) / kTile, ty1 = uint32_t(rows.y) / kTile;
    const uint32_t n_rows = ty1 - ty0 + 1u;
    bool complete = n_rows <= 6u;
    unsigned long long lo = 0ull;
    uint32_t hi = 0u;
    for (uint32_t ty = ty0; ty <= ty1; ++ty) {
      const uint2 span = footprint_row_tiles(mx, my, a, b, c, t, rows, ty, width);
      const uint32_t w = span.y - span.x;
      tiles += w;
      complete = complete && span.x < 1024u && w < 64u;
      if (complete) {
        const uint32_t r = ty - ty0, v = span.x | w << 10;
        if (r < 4u) lo |= static_cast<unsigned long long>(v) << (16u * r);
        else hi |= v << (16u * (r - 4u));
      }
    }
    packed = make_uint4(ty0 | min(n_rows, 255u) << 16 | (complete ? 1u << 31 : 0u), uint32_t(lo), uint32_t(lo >> 32),
                        hi);
  }
  return tiles;
}

// Tile count of the ellipse (train_project.comp:75-81).
__device__ __forceinline__ uint32_t footprint_count(float mx, float my, float a, float b, float c, float t,
                                                    uint32_t width, uint32_t height) {
  const int2 rows = footprint_rows(mx, my, c, t, height);
  uint32_t tiles = 0u;
  if (rows.x <= rows.y) {
    for (uint32_t ty = uint32_t(rows.x) / kTile; ty <= uint32_t(rows.y) / kTile; ++ty) {
      const uint2 span = footprint_row_tiles(mx, my, a, b, c, t, rows, ty, width);
      tiles += span.y - span.x;
    }
  }
  return tiles;
}

// Loss weight of the pixel centred at (px, py) (train_common.glsl:41-45).
__device__ __forceinline__ float pixel_weight(const float4 head, float px, float py) {
  if (head.z <= 0.0f) return 1.0f;
  const float dx = px - head.x, dy = py - head.y;
  const float d = sqrtf(dx * dx + dy * dy) / head.z;
  const float s = clampf((d - 0.8f) / 0.2f, 0.0f, 1.0f);
  return 1.0f + (head.w - 1.0f) * (1.0f - s * s * (3.0f - 2.0f * s));
}

// Pixel of thread `lid` within a 16x16 tile. Each warp covers an 8x4 block, so a
// warp's pixels are close together (the backward pass reduces per warp).
__device__ __forceinline__ uint2 tile_pixel(uint32_t lid) {
  const uint32_t w = lid >> 5, l = lid & 31u;
  return make_uint2((w & 1u) * 8u + (l & 7u), (w >> 1) * 4u + (l >> 3));
}

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }

}  // namespace gsk
