// Loss: SSIM and its gradient (train_ssim.comp:49-142, train_ssim_grad.comp:23-70) per
// 16x16 tile with a 5-pixel halo, and the per-view loss sums.
//
// The L1 part of dL/dC is written by the forward pass. k_ssim stages render and target
// colour of the 26x26 window block in shared memory, blurs the five moments (rows, then
// columns: the separable 11x11 window, sigma 1.5, zero outside the image) and writes the
// SSIM gradient maps A, B, C; k_ssim_grad blurs those back and subtracts
// lambda / (3 pixels) (G*A + 2 x G*B + y G*C) from dL/dC, then refreshes dL/dC . C.
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
  const float ta = float(u >> 24) / 255.0f;
  const float tr[3] = {float(u & 255u) / 255.0f, float((u >> 8) & 255u) / 255.0f, float((u >> 16) & 255u) / 255.0f};
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

__global__ void __launch_bounds__(256) k_ssim(LossArgs a) {
  __shared__ float s_x[3][kWin * kWin];
  __shared__ float s_y[3][kWin * kWin];
  __shared__ float s_h[5][kWin * kTile];
  __shared__ float s_sum[8][2];
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
  for (uint32_t e = lid; e < uint32_t(kWin * kWin); e += 256u) {
    const int gx = ox + int(e % kWin), gy = oy + int(e / kWin);
    const bool in = gx >= 0 && gy >= 0 && gx < int(W) && gy < int(H);
    float3 x = make_float3(0.f, 0.f, 0.f), y = x;
    if (in) {
      const size_t local = size_t(gy) * W + size_t(gx);
      const float4 o = a.rb.pixel_out[pbase + local];
      x = make_float3(o.x, o.y, o.z);
      y = target_colour(f, target[local]);
    }
    s_x[0][e] = x.x; s_x[1][e] = x.y; s_x[2][e] = x.z;
    s_y[0][e] = y.x; s_y[1][e] = y.y; s_y[2][e] = y.z;
  }
  const uint32_t lx = lid % kTile, ly = lid / kTile;
  const uint32_t px = uint32_t(tx) * kTile + lx, py = uint32_t(ty) * kTile + ly;
  const bool inside = px < W && py < H;
  const size_t pix = pbase + size_t(py) * W + px;
  const float w = inside ? a.rb.pixel_out[pix].w : 0.0f;
  const float c1 = f.loss[1], c2 = f.loss[2];
  float A[3], B[3], C[3], ssim_sum = 0.0f, wsum = 0.0f;
  __syncthreads();
  for (int c = 0; c < 3; ++c) {
    for (uint32_t e = lid; e < uint32_t(kWin * kTile); e += 256u) {
      const uint32_t row = e / kTile, col = e % kTile;
      float m0 = 0.f, m1 = 0.f, m2 = 0.f, m3 = 0.f, m4 = 0.f;
#pragma unroll
      for (int k = 0; k <= 2 * kR; ++k) {
        const float wk = c_window[k];
        const float x = s_x[c][row * kWin + col + k], y = s_y[c][row * kWin + col + k];
        m0 += wk * x;
        m1 += wk * y;
        m2 += wk * x * x;
        m3 += wk * y * y;
        m4 += wk * x * y;
      }
      s_h[0][e] = m0;
      s_h[1][e] = m1;
      s_h[2][e] = m2;
      s_h[3][e] = m3;
      s_h[4][e] = m4;
    }
    __syncthreads();
    float mx = 0.f, my = 0.f, exx = 0.f, eyy = 0.f, exy = 0.f;
#pragma unroll
    for (int k = 0; k <= 2 * kR; ++k) {
      const float wk = c_window[k];
      const uint32_t e = (ly + k) * kTile + lx;
      mx += wk * s_h[0][e];
      my += wk * s_h[1][e];
      exx += wk * s_h[2][e];
      eyy += wk * s_h[3][e];
      exy += wk * s_h[4][e];
    }
    const float vx = exx - mx * mx, vy = eyy - my * my, cxy = exy - mx * my;
    const float l = 2.0f * mx * my + c1, cs = 2.0f * cxy + c2;
    const float m = mx * mx + my * my + c1, vv = vx + vy + c2;
    const float inv = 1.0f / (m * vv);
    const float ssim = l * cs * inv;
    const float d_cxy = 2.0f * l * inv;
    const float d_vx = -ssim / vv;
    A[c] = 2.0f * my * cs * inv - ssim * 2.0f * mx / m - 2.0f * mx * d_vx - my * d_cxy;
    B[c] = d_vx;
    C[c] = d_cxy;
    if (inside) {
      ssim_sum += ssim;
      wsum += w * ssim;
    }
    __syncthreads();
  }
  if (inside) {
    a.rb.ssim_maps[pix * 3u] = make_float4(w * A[0], w * A[1], w * A[2], 0.0f);
    a.rb.ssim_maps[pix * 3u + 1u] = make_float4(w * B[0], w * B[1], w * B[2], 0.0f);
    a.rb.ssim_maps[pix * 3u + 2u] = make_float4(w * C[0], w * C[1], w * C[2], 0.0f);
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
    for (int w8 = 0; w8 < 8; ++w8) s += s_sum[w8][lid];
    a.rb.tile_loss[size_t(gt) * 16u + (lid == 0 ? 2u : 4u)] = s;
  }
}

__global__ void __launch_bounds__(256) k_ssim_grad(LossArgs a) {
  __shared__ float s_m[3][kWin * kWin];
  __shared__ float s_h[3][kWin * kTile];
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
  const uint32_t lx = lid % kTile, ly = lid / kTile;
  const uint32_t px = uint32_t(tx) * kTile + lx, py = uint32_t(ty) * kTile + ly;
  const bool inside = px < W && py < H;
  const size_t pix = pbase + size_t(py) * W + px;
  float3 x = make_float3(0.f, 0.f, 0.f), y = x;
  if (inside) {
    const float4 o = a.rb.pixel_out[pix];
    x = make_float3(o.x, o.y, o.z);
    y = target_colour(f, target[size_t(py) * W + px]);
  }
  float ds[3];
  for (int c = 0; c < 3; ++c) {
    for (uint32_t e = lid; e < uint32_t(kWin * kWin); e += 256u) {
      const int gx = ox + int(e % kWin), gy = oy + int(e / kWin);
      const bool in = gx >= 0 && gy >= 0 && gx < int(W) && gy < int(H);
      float m0 = 0.f, m1 = 0.f, m2 = 0.f;
      if (in) {
        const size_t q = (pbase + size_t(gy) * W + size_t(gx)) * 3u;
        const float* maps = reinterpret_cast<const float*>(a.rb.ssim_maps);
        m0 = maps[q * 4u + c];
        m1 = maps[(q + 1u) * 4u + c];
        m2 = maps[(q + 2u) * 4u + c];
      }
      s_m[0][e] = m0;
      s_m[1][e] = m1;
      s_m[2][e] = m2;
    }
    __syncthreads();
    for (uint32_t e = lid; e < uint32_t(kWin * kTile); e += 256u) {
      const uint32_t row = e / kTile, col = e % kTile;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        float sum = 0.0f;
#pragma unroll
        for (int k = 0; k <= 2 * kR; ++k) sum += c_window[k] * s_m[q][row * kWin + col + k];
        s_h[q][e] = sum;
      }
    }
    __syncthreads();
    float g[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
      for (int k = 0; k <= 2 * kR; ++k) g[q] += c_window[k] * s_h[q][(ly + k) * kTile + lx];
    const float xc = c == 0 ? x.x : (c == 1 ? x.y : x.z);
    const float yc = c == 0 ? y.x : (c == 1 ? y.y : y.z);
    ds[c] = g[0] + 2.0f * xc * g[1] + yc * g[2];
    __syncthreads();
  }
  if (inside) {
    float4 pg = a.rb.pixel_grad[pix];
    const float s = f.loss[0] * f.background[3];
    pg.x -= s * ds[0];
    pg.y -= s * ds[1];
    pg.z -= s * ds[2];
    a.rb.pixel_grad[pix] = pg;
    a.rb.pixel_dot[pix] = pg.x * x.x + pg.y * x.y + pg.z * x.z;
  }
}

__global__ void __launch_bounds__(256) k_loss_reduce(const ViewTable* vt, const float* __restrict__ tile_loss,
                                                     double* __restrict__ view_sums) {
  __shared__ double s[8][8];
  const uint32_t v = blockIdx.x;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const uint32_t t0 = vt->tile_base[v], t1 = vt->tile_base[v + 1];
  for (uint32_t t = t0 + threadIdx.x; t < t1; t += 256u)
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] += double(tile_loss[size_t(t) * 16u + k]);
#pragma unroll
  for (int k = 0; k < 8; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if ((threadIdx.x & 31u) == 0u)
#pragma unroll
    for (int k = 0; k < 8; ++k) s[threadIdx.x >> 5][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < 8u) {
    double sum = 0.0;
    for (int w = 0; w < 8; ++w) sum += s[w][threadIdx.x];
    view_sums[v * 8u + threadIdx.x] = sum;
  }
}

}  // namespace

void launch_ssim(const StepPointers& sp, const RasterBuffers& rb, cudaStream_t st) {
  if (sp.tile_cap == 0u) return;
  k_ssim<<<sp.tile_cap, 256, 0, st>>>(LossArgs{sp.frames, sp.vt, rb});
}

void launch_ssim_grad(const StepPointers& sp, const RasterBuffers& rb, cudaStream_t st) {
  if (sp.tile_cap == 0u) return;
  k_ssim_grad<<<sp.tile_cap, 256, 0, st>>>(LossArgs{sp.frames, sp.vt, rb});
}

void launch_loss_reduce(const StepPointers& sp, const float* tile_loss, double* view_sums, cudaStream_t st) {
  if (sp.n_views == 0u) return;
  k_loss_reduce<<<sp.n_views, 256, 0, st>>>(sp.vt, tile_loss, view_sums);
}

}  // namespace gsk
