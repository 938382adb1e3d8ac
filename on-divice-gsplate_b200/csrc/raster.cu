// Tile rasterisation: forward blend (train_forward.comp:59-183) and its adjoint
// (train_common.glsl:215-253; the front-to-back form of train_backward_bucket.glsl:14-16).
//
// Both run one 256-thread block per 16x16 tile of the flattened (view, tile) space, so a
// batch of views of uneven resolution is one launch. Splat records are gathered through
// the sorted pair list into shared memory a batch at a time and read back as broadcasts.
//
// The adjoint keeps no per-fragment state: each pixel walks its splats front to back
// again from T = 1 and R = dL/dC . C_final (pixel_dot, background included), up to its
// last contributor (pixel_count), reproducing the forward's transmittance bit for bit
// (same multiplications). Per splat it needs
//   dL/dalpha_k = T_k (dL/dC . c_k) - R_{k+1} / (1 - alpha_k),  R_{k+1} = R_k - (dL/dC . c_k) alpha_k T_k.
// Each warp sums a splat's 12 gradient values over its 32 pixels with a reduce-scatter
// butterfly (16 shuffles instead of 60 for a tree per value), skipped when no lane of the
// warp touched the splat; the 8 warps' partials are then added in a fixed order, so the
// per-pair gradient is bit-stable. Deterministic mode stores it at the pair's pre-sort
// index (pair_grads, summed per gaussian by train_pair_sum's fixed order); fast mode adds
// it to the gaussian's accumulator with one atomic per value and tile.
#include "gs_kernels.h"

namespace gsk {
namespace {

struct FwdArgs {
  const gs_frame_data* frames;
  ViewTable vt;
  RasterBuffers rb;
  const float4* splat;
};

__device__ __forceinline__ uint32_t pack_unorm(float v) { return uint32_t(clampf(v, 0.0f, 1.0f) * 255.0f + 0.5f); }

__global__ void __launch_bounds__(256) k_raster_fwd(FwdArgs a) {
  __shared__ float4 s_a[256];  // centre xy, opacity, conic a
  __shared__ float4 s_b[256];  // conic b, conic c, red, green
  __shared__ float s_c[256];   // blue
  __shared__ float s_red[8][16];
  __shared__ uint32_t s_max[8];

  const uint32_t gt = blockIdx.x;
  const uint32_t v = view_of_tile(a.vt, gt);
  const gs_frame_data& f = a.frames[v];
  const uint32_t W = f.image[0], H = f.image[1], tiles_x = f.image[2];
  const uint32_t t = gt - a.vt.tile_base[v];
  const uint32_t lid = threadIdx.x, lane = lid & 31u, warp = lid >> 5;
  const uint2 tp = tile_pixel(lid);
  const uint32_t px = (t % tiles_x) * kTile + tp.x, py = (t / tiles_x) * kTile + tp.y;
  const bool inside = px < W && py < H;
  const float cx = float(px) + 0.5f, cy = float(py) + 0.5f;
  const uint2 range = a.rb.ranges[gt];

  bool done = !inside;
  float T = 1.0f, C0 = 0.0f, C1 = 0.0f, C2 = 0.0f;
  uint32_t contributor = 0u, last = 0u;
  for (uint32_t start = range.x; start < range.y; start += 256u) {
    if (__syncthreads_count(done) == 256) break;
    const uint32_t k = start + lid;
    if (k < range.y) {
      const uint32_t g = a.rb.pair_gaussian[a.rb.values[k]];
      const float4 q0 = a.splat[size_t(g) * 3u], q1 = a.splat[size_t(g) * 3u + 1u], q2 = a.splat[size_t(g) * 3u + 2u];
      s_a[lid] = make_float4(q0.x, q0.y, q0.w, q1.x);
      s_b[lid] = make_float4(q1.y, q1.z, q2.x, q2.y);
      s_c[lid] = q2.z;
    }
    __syncthreads();
    const uint32_t n = min(256u, range.y - start);
    for (uint32_t j = 0; j < n && !done; ++j) {
      ++contributor;
      const float4 A = s_a[j];
      const float4 B = s_b[j];
      const float dx = A.x - cx, dy = A.y - cy;
      const float power = -0.5f * (A.w * dx * dx + B.y * dy * dy) - B.x * dx * dy;
      if (power > 0.0f) continue;
      const float alpha = fminf(kMaxAlpha, A.z * __expf(power));
      if (alpha < kMinAlpha) continue;
      const float next_T = T * (1.0f - alpha);
      if (next_T < kMinTransmittance) {
        done = true;
        break;
      }
      const float w = alpha * T;
      C0 += B.z * w;
      C1 += B.w * w;
      C2 += s_c[j] * w;
      T = next_T;
      last = contributor;
    }
  }

  float vals[14];
#pragma unroll
  for (int k = 0; k < 14; ++k) vals[k] = 0.0f;
  if (inside) {
    const size_t pix = size_t(a.vt.pixel_base[v]) + size_t(py) * W + px;
    const float o0 = C0 + T * f.background[0], o1 = C1 + T * f.background[1], o2 = C2 + T * f.background[2];
    float d0 = 0.0f, d1 = 0.0f, d2 = 0.0f, w = 1.0f;
    if (a.rb.target != nullptr) {
      const uint32_t u = a.rb.target[pix];
      const float ta = float(u >> 24) / 255.0f;
      const float tr[3] = {float(u & 255u) / 255.0f, float((u >> 8) & 255u) / 255.0f, float((u >> 16) & 255u) / 255.0f};
      const bool masked = (f.model[3] & GS_FLAG_MASKED_TARGET) != 0u;
      float tc[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float photo = tr[c] * f.exposure[c];
        tc[c] = masked ? f.background[c] * (1.0f - ta) + photo * ta : photo;
      }
      const float e0 = o0 - tc[0], e1 = o1 - tc[1], e2 = o2 - tc[2];
      w = pixel_weight(make_float4(f.head[0], f.head[1], f.head[2], f.head[3]), cx, cy);
      const float s = (1.0f - f.loss[0]) * f.background[3] * w;
      d0 = e0 > 0.0f ? s : (e0 < 0.0f ? -s : 0.0f);
      d1 = e1 > 0.0f ? s : (e1 < 0.0f ? -s : 0.0f);
      d2 = e2 > 0.0f ? s : (e2 < 0.0f ? -s : 0.0f);
      const float l0 = fabsf(e0) + fabsf(e1) + fabsf(e2);
      const float l1 = e0 * e0 + e1 * e1 + e2 * e2;
      vals[0] = l0;
      vals[1] = l1;
      vals[2] = w * l0;
      vals[3] = 3.0f * w;
      const float hx = cx - f.head[0], hy = cy - f.head[1];
      if (f.head[2] > 0.0f && sqrtf(hx * hx + hy * hy) <= f.head[2]) {
        vals[4] = l1;
        vals[5] = 1.0f;
      }
      if (ta > 0.95f && T < 0.05f) {
        vals[6] = C0 * C0;
        vals[7] = C1 * C1;
        vals[8] = C2 * C2;
        vals[9] = 1.0f;
        vals[10] = C0 * tr[0];
        vals[11] = C1 * tr[1];
        vals[12] = C2 * tr[2];
      }
      vals[13] = ta > 0.0f ? 1.0f : 0.0f;
    }
    a.rb.pixel_out[pix] = make_float4(o0, o1, o2, w);
    a.rb.pixel_grad[pix] = make_float4(d0, d1, d2, T);
    a.rb.pixel_count[pix] = last;
    a.rb.image[pix] = pack_unorm(o0) | pack_unorm(o1) << 8 | pack_unorm(o2) << 16 | pack_unorm(1.0f - T) << 24;
    a.rb.pixel_dot[pix] = d0 * o0 + d1 * o1 + d2 * o2;
  }
  // Tile sums in a fixed order: a butterfly per warp, then the 8 warps.
#pragma unroll
  for (int k = 0; k < 14; ++k) {
    float x = vals[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    vals[k] = x;
  }
  const uint32_t wmax = __reduce_max_sync(0xffffffffu, last);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 14; ++k) s_red[warp][k] = vals[k];
    s_max[warp] = wmax;
  }
  __syncthreads();
  if (lid < 16) {
    float s = 0.0f;
    if (lid < 14)
      for (int w8 = 0; w8 < 8; ++w8) s += s_red[w8][lid];
    // Layout of train_forward.comp:18-23 (slots 2 and 4 are the SSIM pass's):
    // values 0, 1 -> slots 0, 1; value 2 -> slot 3; values 3..13 -> slots 5..15.
    float* tl = a.rb.tile_loss + size_t(gt) * 16u;
    if (lid < 14) tl[lid < 2 ? lid : (lid == 2 ? 3 : lid + 2)] = s;
    if (lid == 14) tl[2] = 0.0f;
    if (lid == 15) tl[4] = 0.0f;
  }
  if (lid == 0) {
    uint32_t m = 0u;
    for (int w8 = 0; w8 < 8; ++w8) m = max(m, s_max[w8]);
    a.rb.tile_count[gt] = m;
  }
}

struct BwdArgs {
  const gs_frame_data* frames;
  ViewTable vt;
  RasterBuffers rb;
  const float4* splat;
  float* pair_grads;  // 12 per pre-sort pair (deterministic)
  float* grad2d;      // 12 per g (fast)
  const uint32_t* d_pairs;
  uint32_t accept;
};

template <int BATCH, bool DET>
__global__ void __launch_bounds__(256) k_raster_bwd(BwdArgs a) {
  if (*a.d_pairs > a.accept) return;  // more pairs than stored: the step's update is skipped
  __shared__ float4 s_a[BATCH];
  __shared__ float4 s_b[BATCH];
  __shared__ float s_c[BATCH];
  __shared__ uint32_t s_dst[BATCH];
  __shared__ float s_part[8][BATCH][12];
  __shared__ uint32_t s_wlast[8];

  const uint32_t gt = blockIdx.x;
  const uint32_t v = view_of_tile(a.vt, gt);
  const gs_frame_data& f = a.frames[v];
  const uint32_t W = f.image[0], H = f.image[1], tiles_x = f.image[2];
  const uint32_t t = gt - a.vt.tile_base[v];
  const uint32_t lid = threadIdx.x, lane = lid & 31u, warp = lid >> 5;
  const uint2 tp = tile_pixel(lid);
  const uint32_t px = (t % tiles_x) * kTile + tp.x, py = (t / tiles_x) * kTile + tp.y;
  const bool inside = px < W && py < H;
  const float cx = float(px) + 0.5f, cy = float(py) + 0.5f;
  const uint2 range = a.rb.ranges[gt];
  const uint32_t len = range.y - range.x;
  const uint32_t n = min(len, a.rb.tile_count[gt]);
  if (DET) {
    // Pairs behind the tile's furthest last contributor draw nothing (train_backward_serial.glsl:58-66).
    for (uint32_t k = range.x + n + lid; k < range.y; k += 256u) {
      float4* o = reinterpret_cast<float4*>(a.pair_grads + size_t(a.rb.values[k]) * 12u);
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      o[0] = z;
      o[1] = z;
      o[2] = z;
    }
  }
  if (n == 0u) return;

  float dl0 = 0.0f, dl1 = 0.0f, dl2 = 0.0f, R = 0.0f, T = 1.0f;
  uint32_t last = 0u;
  if (inside) {
    const size_t pix = size_t(a.vt.pixel_base[v]) + size_t(py) * W + px;
    const float4 pg = a.rb.pixel_grad[pix];
    dl0 = pg.x;
    dl1 = pg.y;
    dl2 = pg.z;
    R = a.rb.pixel_dot[pix];
    last = a.rb.pixel_count[pix];
  }
  const uint32_t wlast = __reduce_max_sync(0xffffffffu, last);
  if (lane == 0) s_wlast[warp] = wlast;

  for (uint32_t start = 0; start < n; start += BATCH) {
    __syncthreads();
    if (lid < uint32_t(BATCH) && start + lid < n) {
      const uint32_t pre = a.rb.values[range.x + start + lid];
      const uint32_t g = a.rb.pair_gaussian[pre];
      const float4 q0 = a.splat[size_t(g) * 3u], q1 = a.splat[size_t(g) * 3u + 1u], q2 = a.splat[size_t(g) * 3u + 2u];
      s_a[lid] = make_float4(q0.x, q0.y, q0.w, q1.x);
      s_b[lid] = make_float4(q1.y, q1.z, q2.x, q2.y);
      s_c[lid] = q2.z;
      s_dst[lid] = DET ? pre : g;
    }
    __syncthreads();
    const uint32_t nb = min(uint32_t(BATCH), n - start);
    const uint32_t jmax = wlast > start ? min(nb, wlast - start) : 0u;
    for (uint32_t j = 0; j < jmax; ++j) {
      float c[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) c[k] = 0.0f;
      bool has = false;
      if (start + j + 1u <= last) {
        const float4 A = s_a[j];
        const float4 B = s_b[j];
        const float dx = A.x - cx, dy = A.y - cy;
        const float power = -0.5f * (A.w * dx * dx + B.y * dy * dy) - B.x * dx * dy;
        if (power <= 0.0f) {
          const float G = __expf(power);
          const float raw = A.z * G;
          const float alpha = fminf(kMaxAlpha, raw);
          if (alpha >= kMinAlpha) {
            has = true;
            const float gc = dl0 * B.z + dl1 * B.w + dl2 * s_c[j];
            const float w = alpha * T;
            const float rest = R - gc * w;
            const float one_minus = 1.0f - alpha;
            const float dlda = T * gc - rest / one_minus;
            const bool clamped = raw >= kMaxAlpha;
            const float dop = clamped ? 0.0f : G * dlda;
            const float dpow = clamped ? 0.0f : raw * dlda;
            const float dmx = dpow * -(A.w * dx + B.x * dy);
            const float dmy = dpow * -(B.y * dy + B.x * dx);
            c[0] = dmx;
            c[1] = dmy;
            c[2] = dpow * (-0.5f * dx * dx);
            c[3] = dpow * (-dx * dy);
            c[4] = dpow * (-0.5f * dy * dy);
            c[5] = dop;
            c[6] = w * dl0;
            c[7] = w * dl1;
            c[8] = w * dl2;
            c[9] = fabsf(dmx);
            c[10] = fabsf(dmy);
            T = T * one_minus;
            R = rest;
          }
        }
      }
      if (__any_sync(0xffffffffu, has)) {
        // Reduce-scatter: lane l ends with the warp sum of value (l >> 1).
        const bool b4 = lane & 16u, b3 = lane & 8u, b2 = lane & 4u, b1 = lane & 2u;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float send = b4 ? c[i] : c[i + 8];
          const float keep = b4 ? c[i + 8] : c[i];
          c[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float send = b3 ? c[i] : c[i + 4];
          const float keep = b3 ? c[i + 4] : c[i];
          c[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
        }
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const float send = b2 ? c[i] : c[i + 2];
          const float keep = b2 ? c[i + 2] : c[i];
          c[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
        }
        {
          const float send = b1 ? c[0] : c[1];
          const float keep = b1 ? c[1] : c[0];
          c[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
        }
        c[0] += __shfl_xor_sync(0xffffffffu, c[0], 1);
        if ((lane & 1u) == 0u && (lane >> 1) < 12u) s_part[warp][j][lane >> 1] = c[0];
      } else if (lane < 12u) {
        s_part[warp][j][lane] = 0.0f;
      }
    }
    __syncthreads();
    for (uint32_t idx = lid; idx < nb * 12u; idx += 256u) {
      const uint32_t j = idx / 12u, k = idx - j * 12u;
      float s = 0.0f;
#pragma unroll
      for (int w8 = 0; w8 < 8; ++w8)
        if (start + j < s_wlast[w8]) s += s_part[w8][j][k];
      if (DET) {
        a.pair_grads[size_t(s_dst[j]) * 12u + k] = s;
      } else if (s != 0.0f) {
        atomicAdd(a.grad2d + size_t(s_dst[j]) * 12u + k, s);
      }
    }
  }
}

}  // namespace

void launch_raster_forward(const StepPointers& sp, const ViewBuffers& vb, const RasterBuffers& rb, cudaStream_t st) {
  if (sp.total_tiles == 0u) return;
  FwdArgs a{sp.frames, sp.vt, rb, vb.splat};
  k_raster_fwd<<<sp.total_tiles, 256, 0, st>>>(a);
}

void launch_raster_backward(const StepPointers& sp, const ViewBuffers& vb, const RasterBuffers& rb,
                            float4* pair_grads, bool deterministic, int batch, const uint32_t* d_pairs,
                            uint32_t accept, cudaStream_t st) {
  if (sp.total_tiles == 0u) return;
  BwdArgs a{sp.frames, sp.vt, rb, vb.splat, reinterpret_cast<float*>(pair_grads),
            reinterpret_cast<float*>(vb.grad2d), d_pairs, accept};
  if (batch <= 32) {
    if (deterministic) k_raster_bwd<32, true><<<sp.total_tiles, 256, 0, st>>>(a);
    else k_raster_bwd<32, false><<<sp.total_tiles, 256, 0, st>>>(a);
  } else {
    if (deterministic) k_raster_bwd<64, true><<<sp.total_tiles, 256, 0, st>>>(a);
    else k_raster_bwd<64, false><<<sp.total_tiles, 256, 0, st>>>(a);
  }
}

}  // namespace gsk
