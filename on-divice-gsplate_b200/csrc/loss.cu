// Loss: SSIM and its gradient (train_ssim.comp:49-142, train_ssim_grad.comp:23-70) per
// 16x16 tile with a 5-pixel halo, and the per-view loss sums.
//
// The L1 part of dL/dC is written by the forward pass. k_ssim stages render and target
// colour of the 26x26 window block in shared memory, blurs the five moments (rows, then
// columns: the separable 11x11 window, sigma 1.5, zero outside the image) and writes the
// SSIM gradient maps A, B, C; k_ssim_grad blurs those back and subtracts
// lambda / (3 pixels) (G*A + 2 x G*B + y G*C) from dL/dC, then refreshes dL/dC . C.
//
// Both blurs are register-blocked: a thread produces 4 consecutive outputs of a row (or
// column) from the 14 inputs it loads once (8 from 18 in k_ssim_grad, whose blurs carry
// one plane), so shared-memory traffic per output is 3.5 (2.25) loads per plane instead of
// 11, and sums run over the taps in window order. The row
// blur's results are kept column-major (26 rows of a column contiguous): a warp's stores
// (8 rows x 4 runs) then fall on 32 different banks, and the column blur reads its 14
// rows as 7 aligned 8-byte loads.
#include "gs_kernels.h"

namespace gsk {
namespace {

constexpr int kR = 5;
constexpr int kWin = kTile + 2 * kR;  // 26
__constant__ float c_window[11] = {0.001028380f, 0.007598758f, 0.036000772f, 0.109360690f,
                                   0.213005538f, 0.266011725f, 0.213005538f, 0.109360690f,
                                   0.036000772f, 0.007598758f, 0.001028380f};

struct LossArgs {
  const gs_frame_data* frames;
  const ViewTable* vt;
  RasterBuffers rb;
};

// The target colour the loss compares against (train_forward.comp:124-126).
__device__ __forceinline__ float3 target_colour(const gs_frame_data& f, uint32_t u) {
  constexpr float k = 1.0f / 255.0f;
  const float ta = float(u >> 24) * k;
  const float tr[3] = {float(u & 255u) * k, float((u >> 8) & 255u) * k, float((u >> 16) & 255u) * k};
  const bool masked = (f.model[3] & GS_FLAG_MASKED_TARGET) != 0u;
  float tc[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float photo = tr[c] * f.exposure[c];
    tc[c] = masked ? f.background[c] * (1.0f - ta) + photo * ta : photo;
  }
  return make_float3(tc[0], tc[1], tc[2]);
}

// train_ssim.comp:35-47: no splat and no subject pixel in the 3x3 tiles around.
__device__ bool background_only(const LossArgs& a, const gs_frame_data& f, uint32_t v, int tx, int ty) {
  if ((f.model[3] & GS_FLAG_MASKED_TARGET) == 0u) return false;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx) {
      const int nx = tx + dx, ny = ty + dy;
      if (nx < 0 || ny < 0 || nx >= int(f.image[2]) || ny >= int(f.image[3])) continue;
      const uint32_t t = a.vt->tile_base[v] + uint32_t(ny) * f.image[2] + uint32_t(nx);
      const uint2 r = a.rb.ranges[t];
      if (r.y > r.x || a.rb.tile_loss[size_t(t) * 16u + 15u] > 0.0f) return false;
    }
  return true;
}

constexpr int kRun = 4;                 // outputs per thread and blur
constexpr int kSpan = kRun + 2 * kR;    // inputs a thread loads: 14
constexpr int kQuads = kTile / kRun;    // 4
constexpr int kS = kWin + 1;            // row stride of a staged plane (odd: at most 2-way conflicts)
constexpr int kPlane = kWin * kS;       // 702
constexpr int kHRow = kWin * kTile;     // one plane after the row blur: 16 columns x 26 rows, column-major
constexpr int kHPlane = kHRow + 16;     // padded so neighbouring planes fall on other banks (even: 8-byte aligned)
constexpr int kAbc = kTilePixels + 16;  // stride of the per-pixel planes after the column blur
// Threads of an SSIM block: ten warps, so the row blur of k_ssim (312 runs) takes one round
// and those of k_ssim_grad (468 row runs, 288 column runs of 8) two and one; the per-pixel
// phases use the first 256.
constexpr uint32_t kLossThreads = 320;
constexpr uint32_t kLossWarps = kLossThreads / 32;
constexpr uint32_t kWindowLoads = (kWin * kWin + kLossThreads - 1) / kLossThreads;  // 3 window pixels a thread

// Blur of 4 consecutive outputs from `src` (14 inputs, `stride` apart) into out[4].
__device__ __forceinline__ void blur4(const float x[kSpan], float out[kRun]) {
#pragma unroll
  for (int o = 0; o < kRun; ++o) {
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k <= 2 * kR; ++k) sum += c_window[k] * x[o + k];
    out[o] = sum;
  }
}

// Column blur: 14 contiguous inputs at an 8-byte-aligned address.
__device__ __forceinline__ void blur_column(const float* src, float out[kRun]) {
  float x[kSpan];
  const float2* s2 = reinterpret_cast<const float2*>(src);
#pragma unroll
  for (int k = 0; k < kSpan / 2; ++k) {
    const float2 v = s2[k];
    x[2 * k] = v.x;
    x[2 * k + 1] = v.y;
  }
  blur4(x, out);
}

// The gradient kernel blurs single planes, so a thread can carry 8 outputs of a run (18
// loads for 8 outputs, 2.25 per output) without running out of registers.
constexpr int kRun8 = 8;
constexpr int kSpan8 = kRun8 + 2 * kR;  // 18
constexpr int kRuns8 = kTile / kRun8;   // 2

__device__ __forceinline__ void blur8(const float x[kSpan8], float out[kRun8]) {
#pragma unroll
  for (int o = 0; o < kRun8; ++o) {
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k <= 2 * kR; ++k) sum += c_window[k] * x[o + k];
    out[o] = sum;
  }
}

__global__ void __launch_bounds__(kLossThreads) k_ssim(LossArgs a) {
  // s_buf: render rgb and target rgb planes of the window (26 x kS each); after the row
  // blur it holds A, B, C and SSIM per channel for the tile's 256 pixels.
  __shared__ float s_buf[6 * kPlane];
  __shared__ __align__(16) float s_h[3 * 5 * kHPlane];  // [channel][moment] after the row blur
  __shared__ float s_sum[kLossWarps][2];
  const uint32_t gt = blockIdx.x;
  if (gt >= a.vt->total_tiles) return;
  const uint32_t v = view_of_tile(a.vt, gt);
  const gs_frame_data& f = a.frames[v];
  const uint32_t* target = a.vt->target[v];
  if (target == nullptr) return;
  const uint32_t W = f.image[0], H = f.image[1];
  const uint32_t t = gt - a.vt->tile_base[v];
  const int tx = int(t % f.image[2]), ty = int(t / f.image[2]);
  const uint32_t lid = threadIdx.x;
  if (background_only(a, f, v, tx, ty)) {
    if (lid == 0) {
      const uint32_t sx = min(kTile, W - uint32_t(tx) * kTile), sy = min(kTile, H - uint32_t(ty) * kTile);
      float* tl = a.rb.tile_loss + size_t(gt) * 16u;
      tl[2] = 3.0f * float(sx * sy);  // SSIM 1 per pixel and channel
      tl[4] = tl[5];
    }
    return;
  }
  const size_t pbase = a.vt->pixel_base[v];
  const int ox = tx * int(kTile) - kR, oy = ty * int(kTile) - kR;
  // Each thread's (up to) three window pixels, all loads issued before the first store.
  float4 xo[kWindowLoads];
  uint32_t yt[kWindowLoads];
  bool in_image[kWindowLoads];
#pragma unroll
  for (uint32_t r = 0; r < kWindowLoads; ++r) {
    const uint32_t e = lid + r * kLossThreads;
    const uint32_t row = e / kWin, col = e % kWin;
    const int gx = ox + int(col), gy = oy + int(row);
    const bool in = e < uint32_t(kWin * kWin) && gx >= 0 && gy >= 0 && gx < int(W) && gy < int(H);
    xo[r] = make_float4(0.f, 0.f, 0.f, 0.f);
    yt[r] = 0u;
    in_image[r] = in;
    if (in) {
      const size_t local = size_t(gy) * W + size_t(gx);
      xo[r] = a.rb.pixel_out[pbase + local];
      yt[r] = target[local];
    }
  }
#pragma unroll
  for (uint32_t r = 0; r < kWindowLoads; ++r) {
    const uint32_t e = lid + r * kLossThreads;
    if (e >= uint32_t(kWin * kWin)) break;
    const float3 y = in_image[r] ? target_colour(f, yt[r]) : make_float3(0.f, 0.f, 0.f);
    const uint32_t at = (e / kWin) * kS + e % kWin;
    s_buf[at] = xo[r].x;
    s_buf[kPlane + at] = xo[r].y;
    s_buf[2 * kPlane + at] = xo[r].z;
    s_buf[3 * kPlane + at] = y.x;
    s_buf[4 * kPlane + at] = y.y;
    s_buf[5 * kPlane + at] = y.z;
  }
  __syncthreads();
  // Row blur of the five moments: 3 channels x 26 rows x 4 runs.
  for (uint32_t e = lid; e < 3u * kWin * kQuads; e += kLossThreads) {
    const uint32_t q = e % kQuads, row = (e / kQuads) % kWin, c = e / (kQuads * kWin);
    const float* xs = s_buf + c * kPlane + row * kS + q * kRun;
    const float* ys = s_buf + (3u + c) * kPlane + row * kS + q * kRun;
    // The inputs and their products, once per loaded pixel.
    float x[kSpan], y[kSpan], xx[kSpan], yy[kSpan], xy[kSpan];
#pragma unroll
    for (int k = 0; k < kSpan; ++k) {
      x[k] = xs[k];
      y[k] = ys[k];
      xx[k] = x[k] * x[k];
      yy[k] = y[k] * y[k];
      xy[k] = x[k] * y[k];
    }
    float* h = s_h + c * 5u * kHPlane + (q * kRun) * kWin + row;  // column q * 4 + o, row `row`
#pragma unroll
    for (int o = 0; o < kRun; ++o) {
      float m0 = 0.f, m1 = 0.f, m2 = 0.f, m3 = 0.f, m4 = 0.f;
#pragma unroll
      for (int k = 0; k <= 2 * kR; ++k) {
        const float wk = c_window[k];
        m0 = fmaf(wk, x[o + k], m0);
        m1 = fmaf(wk, y[o + k], m1);
        m2 = fmaf(wk, xx[o + k], m2);
        m3 = fmaf(wk, yy[o + k], m3);
        m4 = fmaf(wk, xy[o + k], m4);
      }
      h[o * kWin] = m0;
      h[kHPlane + o * kWin] = m1;
      h[2 * kHPlane + o * kWin] = m2;
      h[3 * kHPlane + o * kWin] = m3;
      h[4 * kHPlane + o * kWin] = m4;
    }
  }
  __syncthreads();
  // Column blur and the SSIM terms: 3 channels x 16 columns x 4 runs of 4 pixels.
  float* s_abc = s_buf;  // [A, B, C, SSIM][channel][kAbc]
  const float c1 = f.loss[1], c2 = f.loss[2];
  if (lid < 3u * kTile * kQuads) {
    const uint32_t col = lid % kTile, c = (lid / kTile) % 3u, q = lid / (3u * kTile);
    const float* h = s_h + c * 5u * kHPlane + col * kWin + q * kRun;
    float mom[5][kRun];
#pragma unroll
    for (int j = 0; j < 5; ++j) blur_column(h + j * kHPlane, mom[j]);
#pragma unroll
    for (int o = 0; o < kRun; ++o) {
      const float mx = mom[0][o], my = mom[1][o], exx = mom[2][o], eyy = mom[3][o], exy = mom[4][o];
      const float vx = exx - mx * mx, vy = eyy - my * my, cxy = exy - mx * my;
      const float l = 2.0f * mx * my + c1, cs = 2.0f * cxy + c2;
      const float m = mx * mx + my * my + c1, vv = vx + vy + c2;
      // One reciprocal: 1/(m vv), 1/vv = m/(m vv), 1/m = vv/(m vv).
      const float inv = __fdividef(1.0f, m * vv);
      const float ssim = l * cs * inv;
      const float d_cxy = 2.0f * l * inv;
      const float d_vx = -ssim * (m * inv);
      const uint32_t pixel = (q * kRun + o) * kTile + col;
      s_abc[c * kAbc + pixel] =
          2.0f * my * cs * inv - ssim * 2.0f * mx * (vv * inv) - 2.0f * mx * d_vx - my * d_cxy;
      s_abc[(3u + c) * kAbc + pixel] = d_vx;
      s_abc[(6u + c) * kAbc + pixel] = d_cxy;
      s_abc[(9u + c) * kAbc + pixel] = ssim;
    }
  }
  __syncthreads();
  const uint32_t lx = lid % kTile, ly = lid / kTile;
  const uint32_t px = uint32_t(tx) * kTile + lx, py = uint32_t(ty) * kTile + ly;
  const bool inside = lid < kTilePixels && px < W && py < H;
  const size_t pix = pbase + size_t(py) * W + px;
  float ssim_sum = 0.0f, wsum = 0.0f;
  if (inside) {
    const float w = a.rb.pixel_out[pix].w;
    float A[3], B[3], C[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      A[c] = s_abc[c * kAbc + lid];
      B[c] = s_abc[(3 + c) * kAbc + lid];
      C[c] = s_abc[(6 + c) * kAbc + lid];
      const float ssim = s_abc[(9 + c) * kAbc + lid];
      ssim_sum += ssim;
      wsum += w * ssim;
    }
    a.rb.ssim_maps[pix * 2u] = make_float4(w * A[0], w * A[1], w * A[2], w * B[0]);
    a.rb.ssim_maps[pix * 2u + 1u] = make_float4(w * B[1], w * B[2], w * C[0], w * C[1]);
    a.rb.ssim_last[pix] = w * C[2];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ssim_sum += __shfl_xor_sync(0xffffffffu, ssim_sum, o);
    wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
  }
  if ((lid & 31u) == 0u) {
    s_sum[lid >> 5][0] = ssim_sum;
    s_sum[lid >> 5][1] = wsum;
  }
  __syncthreads();
  if (lid < 2u) {
    float s = 0.0f;
    for (uint32_t w8 = 0; w8 < kLossWarps; ++w8) s += s_sum[w8][lid];
    a.rb.tile_loss[size_t(gt) * 16u + (lid == 0 ? 2u : 4u)] = s;
  }
}

__global__ void __launch_bounds__(kLossThreads) k_ssim_grad(LossArgs a) {
  // s_m: the 9 planes (A, B, C x rgb) of the window; after the row blur it holds the
  // 9 blurred planes of the tile's 256 pixels.
  __shared__ float s_m[9 * kPlane];
  __shared__ __align__(16) float s_h[9 * kHPlane];
  const uint32_t gt = blockIdx.x;
  if (gt >= a.vt->total_tiles) return;
  const uint32_t v = view_of_tile(a.vt, gt);
  const gs_frame_data& f = a.frames[v];
  const uint32_t* target = a.vt->target[v];
  if (target == nullptr) return;
  // Without splats in the tile nothing reads its pixels' gradients (masked targets).
  const uint2 own = a.rb.ranges[gt];
  if ((f.model[3] & GS_FLAG_MASKED_TARGET) != 0u && own.y <= own.x) return;
  const uint32_t W = f.image[0], H = f.image[1];
  const uint32_t t = gt - a.vt->tile_base[v];
  const int tx = int(t % f.image[2]), ty = int(t / f.image[2]);
  const uint32_t lid = threadIdx.x;
  const size_t pbase = a.vt->pixel_base[v];
  const int ox = tx * int(kTile) - kR, oy = ty * int(kTile) - kR;
  // The thread's own pixel's inputs of the last phase, loaded now so that their latency
  // hides behind the blurs.
  const uint32_t lx = lid % kTile, ly = lid / kTile;
  const uint32_t px = uint32_t(tx) * kTile + lx, py = uint32_t(ty) * kTile + ly;
  const bool mine = lid < kTilePixels && px < W && py < H;
  const size_t pix = pbase + size_t(py) * W + px;
  float4 o = make_float4(0.f, 0.f, 0.f, 0.f), pg = o;
  uint32_t own_target = 0u;
  if (mine) {
    o = a.rb.pixel_out[pix];
    pg = a.rb.pixel_grad[pix];
    own_target = target[size_t(py) * W + px];
  }
  // Each thread's (up to) three window pixels: every load issued before the first store,
  // so their latencies overlap instead of adding up.
  float4 m0[kWindowLoads], m1[kWindowLoads];
  float m2[kWindowLoads];
#pragma unroll
  for (uint32_t r = 0; r < kWindowLoads; ++r) {
    const uint32_t e = lid + r * kLossThreads;
    const uint32_t row = e / kWin, col = e % kWin;
    const int gx = ox + int(col), gy = oy + int(row);
    const bool in = e < uint32_t(kWin * kWin) && gx >= 0 && gy >= 0 && gx < int(W) && gy < int(H);
    m0[r] = make_float4(0.f, 0.f, 0.f, 0.f);
    m1[r] = m0[r];
    m2[r] = 0.0f;
    if (in) {
      const size_t q = pbase + size_t(gy) * W + size_t(gx);
      m0[r] = a.rb.ssim_maps[q * 2u];
      m1[r] = a.rb.ssim_maps[q * 2u + 1u];
      m2[r] = a.rb.ssim_last[q];
    }
  }
#pragma unroll
  for (uint32_t r = 0; r < kWindowLoads; ++r) {
    const uint32_t e = lid + r * kLossThreads;
    if (e >= uint32_t(kWin * kWin)) break;
    // Planes A rgb, B rgb, C rgb.
    const uint32_t at = (e / kWin) * kS + e % kWin;
    s_m[at] = m0[r].x;
    s_m[kPlane + at] = m0[r].y;
    s_m[2 * kPlane + at] = m0[r].z;
    s_m[3 * kPlane + at] = m0[r].w;
    s_m[4 * kPlane + at] = m1[r].x;
    s_m[5 * kPlane + at] = m1[r].y;
    s_m[6 * kPlane + at] = m1[r].z;
    s_m[7 * kPlane + at] = m1[r].w;
    s_m[8 * kPlane + at] = m2[r];
  }
  __syncthreads();
  // Row blur: 9 planes x 26 rows x 2 runs of 8.
  for (uint32_t e = lid; e < 9u * kWin * kRuns8; e += kLossThreads) {
    const uint32_t q = e % kRuns8, row = (e / kRuns8) % kWin, p = e / (kRuns8 * kWin);
    const float* src = s_m + p * kPlane + row * kS + q * kRun8;
    float x[kSpan8], out[kRun8];
#pragma unroll
    for (int k = 0; k < kSpan8; ++k) x[k] = src[k];
    blur8(x, out);
#pragma unroll
    for (int o = 0; o < kRun8; ++o) s_h[p * kHPlane + (q * kRun8 + o) * kWin + row] = out[o];
  }
  __syncthreads();
  // Column blur: 9 planes x 16 columns x 2 runs of 8 (18 contiguous inputs, 8-byte loads).
  float* s_g = s_m;  // [plane][kAbc]
  for (uint32_t e = lid; e < 9u * kTile * kRuns8; e += kLossThreads) {
    const uint32_t col = e % kTile, p = (e / kTile) % 9u, q = e / (9u * kTile);
    const float2* src = reinterpret_cast<const float2*>(s_h + p * kHPlane + col * kWin + q * kRun8);
    float x[kSpan8], out[kRun8];
#pragma unroll
    for (int k = 0; k < kSpan8 / 2; ++k) {
      const float2 v = src[k];
      x[2 * k] = v.x;
      x[2 * k + 1] = v.y;
    }
    blur8(x, out);
#pragma unroll
    for (int o = 0; o < kRun8; ++o) s_g[p * kAbc + (q * kRun8 + o) * kTile + col] = out[o];
  }
  __syncthreads();
  if (!mine) return;
  const float3 y = target_colour(f, own_target);
  const float xs[3] = {o.x, o.y, o.z}, ys[3] = {y.x, y.y, y.z};
  float ds[3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
    ds[c] = s_g[c * kAbc + lid] + 2.0f * xs[c] * s_g[(3 + c) * kAbc + lid] + ys[c] * s_g[(6 + c) * kAbc + lid];
  const float s = f.loss[0] * f.background[3];
  pg.x -= s * ds[0];
  pg.y -= s * ds[1];
  pg.z -= s * ds[2];
  a.rb.pixel_grad[pix] = pg;
  a.rb.pixel_dot[pix] = pg.x * o.x + pg.y * o.y + pg.z * o.z;
}

// The 16 tile sums of each view (Trainer::read_slot, trainer.cpp:778-795), in double and
// a fixed order: kLossParts blocks per view sum consecutive slices of the view's tiles
// (k_loss_partial), then one warp per view adds the slices in order (k_loss_final) into
// view_sums[v * stride + 0..15]. The slices depend only on the view's own tile count, so
// a view's sums do not depend on the other views of the step.
__global__ void __launch_bounds__(256) k_loss_partial(const ViewTable* vt, const float* __restrict__ tile_loss,
                                                      double* __restrict__ parts) {
  __shared__ double s[8][16];
  const uint32_t v = blockIdx.x / kLossParts, part = blockIdx.x % kLossParts;
  const uint32_t t0 = vt->tile_base[v], t1 = vt->tile_base[v + 1];
  const uint32_t chunk = (t1 - t0 + kLossParts - 1u) / kLossParts;
  const uint32_t first = min(t1, t0 + part * chunk), last = min(t1, first + chunk);
  double acc[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) acc[k] = 0.0;
  for (uint32_t t = first + threadIdx.x; t < last; t += 256u) {
    const float4* row = reinterpret_cast<const float4*>(tile_loss + size_t(t) * 16u);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 x = row[q];
      acc[4 * q] += double(x.x);
      acc[4 * q + 1] += double(x.y);
      acc[4 * q + 2] += double(x.z);
      acc[4 * q + 3] += double(x.w);
    }
  }
#pragma unroll
  for (int k = 0; k < 16; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if ((threadIdx.x & 31u) == 0u)
#pragma unroll
    for (int k = 0; k < 16; ++k) s[threadIdx.x >> 5][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < 16u) {
    double sum = 0.0;
    for (int w = 0; w < 8; ++w) sum += s[w][threadIdx.x];
    parts[(size_t(v) * kLossParts + part) * 16u + threadIdx.x] = sum;
  }
}

__global__ void __launch_bounds__(32) k_loss_final(const double* __restrict__ parts, double* __restrict__ view_sums,
                                                   uint32_t stride) {
  const uint32_t v = blockIdx.x;
  if (threadIdx.x >= 16u) return;
  double sum = 0.0;
  for (uint32_t part = 0; part < kLossParts; ++part) sum += parts[(size_t(v) * kLossParts + part) * 16u + threadIdx.x];
  view_sums[size_t(v) * stride + threadIdx.x] = sum;
}

}  // namespace

void launch_ssim(const StepPointers& sp, const RasterBuffers& rb, cudaStream_t st) {
  if (sp.tile_cap == 0u) return;
  k_ssim<<<sp.tile_cap, kLossThreads, 0, st>>>(LossArgs{sp.frames, sp.vt, rb});
}

void launch_ssim_grad(const StepPointers& sp, const RasterBuffers& rb, cudaStream_t st) {
  if (sp.tile_cap == 0u) return;
  k_ssim_grad<<<sp.tile_cap, kLossThreads, 0, st>>>(LossArgs{sp.frames, sp.vt, rb});
}

void launch_loss_reduce(const StepPointers& sp, const float* tile_loss, double* view_sums, uint32_t stride,
                        double* parts, cudaStream_t st) {
  if (sp.n_views == 0u) return;
  k_loss_partial<<<sp.n_views * kLossParts, 256, 0, st>>>(sp.vt, tile_loss, parts);
  k_loss_final<<<sp.n_views, 32, 0, st>>>(parts, view_sums, stride);
}

}  // namespace gsk
