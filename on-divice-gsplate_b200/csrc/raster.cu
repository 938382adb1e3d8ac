// Tile rasterisation: forward blend (train_forward.comp:59-183) and its adjoint
// (train_common.glsl:215-253; the front-to-back form of train_backward_bucket.glsl:14-16).
//
// Both work on 16x16 tiles of the flattened (view, tile) space, taken from an atomic
// queue, so a batch of views of uneven resolution is one launch. Each thread owns PX
// pixels (1, 2 or 4) of a tile, stacked 4 rows apart, so a warp covers an 8 x 4PX block.
// Splat records are gathered through the sorted pair list into shared memory a round at a
// time; a warp ballots which staged splats' footprint ellipses reach its block and walks
// only those, in order (a culled splat is one every pixel of the block would skip anyway).
// The default kernels (raster_fwd_split, raster_bwd_split) make each warp's block its own
// work item, staging its own rounds; the block kernels (raster_fwd_tile, raster_bwd_tile)
// share a round between a tile's warps and serve asynchronous staging and the
// deterministic backward.
//
// The adjoint keeps no per-fragment state: each pixel walks its splats front to back
// again from T = 1 and R = dL/dC . C_final (pixel_dot, background included), up to its
// last contributor (pixel_count), reproducing the forward's transmittance bit for bit
// (same multiplications). Per splat it needs
//   dL/dalpha_k = T_k (dL/dC . c_k) - R_{k+1} / (1 - alpha_k),  R_{k+1} = R_k - (dL/dC . c_k) alpha_k T_k.
// A thread adds its PX pixels' gradients in registers (splat_adjoint); its warp then sums
// the splat's values over its lanes, skipped when no lane touched the splat.
// - Deterministic mode (raster_bwd_tile): the warps of a tile share each staged round; a
//   warp sums a splat's 11 values with a reduce-scatter butterfly (13 shuffles), the warps'
//   partials are added in a fixed order, and the pair's gradient is stored at its pre-sort
//   index (pair_grads, summed per gaussian by train_pair_sum's fixed order): bit-stable.
// - Fast mode (raster_bwd_split): each warp works on its own block of a tile, stages its
//   own rounds and stops at its own last contributor; it sums 9 values through shared
//   memory, and the lane that staged the splat adds them to the gaussian's accumulator with
//   two 16-byte vector atomics (red.global.add.v4.f32) and one scalar. The 9 values a lane
//   contributes are its raw sums, before the splat's opacity and conic factors, which are
//   applied once per splat after the warp sum (raw_to_grads) instead of once per lane and
//   visit. It leaves out the |dL/dmean2d| sums (pair values 9 and 10): they feed only the
//   densify statistic stats.w, which no densify decision reads
//   (train_densify_mark.comp:22-57 uses x, y, z).
// - backward_pixels = 8 (raster_bwd_warp_tile): one warp per whole tile, either mode.
#include "gs_kernels.h"

namespace gsk {
namespace {

struct RasterArgs {
  const gs_frame_data* frames;
  const ViewTable* vt;
  uint32_t* queue;  // work-queue counter of this pass
  RasterBuffers rb;
  const float4* splat;
  const float4* foot;
  float* pair_grads;  // 12 per pre-sort pair (deterministic backward)
  float* grad2d;      // 12 per g (fast backward)
  const uint32_t* d_pairs;
  uint32_t accept;
  unsigned long long* contributions;  // counting forward: pixel-splat evaluations that blend
};

__device__ __forceinline__ uint32_t pack_unorm(float v) { return uint32_t(clampf(v, 0.0f, 1.0f) * 255.0f + 0.5f); }

// A staged splat, in three float4s:
//   A = (centre x, centre y, opacity, ha)   B = (hb, hc, red, green)   C = (blue, limit, kz, kw)
// with the conic (a, b, c) scaled to the base-2 exponent: for the offset d = centre - pixel,
//   E(d) = ha dx^2 + hb dx dy + hc dy^2 = log2(e) power(d),   power = -(a dx^2 + c dy^2)/2 - b dx dy,
// (ha, hb, hc) = -log2(e) (a/2, b, c/2), so alpha = min(0.99, opacity 2^E). Both passes
// evaluate E, alpha and the transmittance with the same operations in the same order
// (fmaf and the non-contracting _rn forms), so the backward reproduces the forward's
// transmittance bit for bit.
//
// Culling: a pixel contributes only if alpha >= 1/255, i.e. Q(d) = -2 power(d) <= 2 ln(255
// opacity); the footprint threshold (train_common.glsl:169-172) already exceeds that, and
// `limit` adds 2^-10 relative and absolute on top (far above the rounding of Q and of the
// fast exponential), stored as the matching bound on E: E >= -log2(e)/2 limit. kz = -b/c and
// kw = -b/a locate the maximum of E along a vertical and a horizontal edge.
constexpr float kLog2e = 1.4426950408889634f;

__device__ __forceinline__ void stage_splat(float4 q0, float4 q1, float4 q2, float threshold, float4& A, float4& B,
                                            float4& C) {
  const float a = q1.x, b = q1.y, c = q1.z;
  A = make_float4(q0.x, q0.y, q0.w, __fmul_rn(a, -0.5f * kLog2e));
  B = make_float4(__fmul_rn(b, -kLog2e), __fmul_rn(c, -0.5f * kLog2e), q2.x, q2.y);
  const float limit = threshold * 1.0009765625f + 0.0009765625f;
  C = make_float4(q2.z, limit * (-0.5f * kLog2e), -__fdividef(b, c), -__fdividef(b, a));
}

// The base-2 exponent at offset (dx, dy); e0 = ha dx dx and e1 = hb dx are per splat and lane.
__device__ __forceinline__ float splat_exponent(float e0, float e1, float hc, float dy) {
  return fmaf(fmaf(hc, dy, e1), dy, e0);
}

__device__ __forceinline__ float exp2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Asynchronous 16-byte global -> shared copies (cp.async, cached in L2 only), grouped per
// staged round: a round's copies are committed as one group, and waiting for all but the
// newest group leaves the next round in flight while the current one is consumed.
__device__ __forceinline__ void copy_async16(void* smem, const void* gmem) {
  const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void copy_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void copy_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
}

// Raw splat records of a staged round, component-major: q[0..2][slot] are the gaussian's
// three splat float4s, q[3][slot] its footprint float4 (whose w is the threshold).
template <int N>
struct RawRound {
  float4 q[4][N];
};
__device__ __forceinline__ void fetch_record_async(float4* q0, float4* q1, float4* q2, float4* qf, const float4* splat,
                                                   const float4* foot, uint32_t g) {
  copy_async16(q0, splat + size_t(g) * 3u);
  copy_async16(q1, splat + size_t(g) * 3u + 1u);
  copy_async16(q2, splat + size_t(g) * 3u + 2u);
  copy_async16(qf, foot + g);
}

// Whether a staged splat's footprint ellipse reaches a pixel centre of the w x h block
// whose first centre is (x0, y0): the maximum of the concave E over the block's rectangle
// is 0 when the centre lies inside, else it lies on an edge facing the centre, at the
// unconstrained maximiser along that edge clamped to the edge.
__device__ __forceinline__ bool block_reached(float4 A, float4 B, float4 C, float x0, float y0, float h,
                                              float w = 8.0f) {
  const float dx0 = x0 - A.x, dx1 = dx0 + (w - 1.0f), dy0 = y0 - A.y, dy1 = dy0 + (h - 1.0f);
  const float ex = dx0 > 0.0f ? dx0 : fminf(dx1, 0.0f);  // facing vertical edge (0: none)
  const float ey = dy0 > 0.0f ? dy0 : fminf(dy1, 0.0f);  // facing horizontal edge (0: none)
  const float ha = A.w, hb = B.x, hc = B.y;
  const float ty = fminf(fmaxf(C.z * ex, dy0), dy1);
  const float tx = fminf(fmaxf(C.w * ey, dx0), dx1);
  const float ev = ex != 0.0f ? ex * (ha * ex + hb * ty) + hc * ty * ty : -3.0e38f;
  const float eh = ey != 0.0f ? tx * (ha * tx + hb * ey) + hc * ey * ey : -3.0e38f;
  const float e = (ex == 0.0f && ey == 0.0f) ? 0.0f : fmaxf(ev, eh);
  return e >= C.y;
}

// Reduce-scatter of 12 slots (11 values and a zero) over a warp: after the exchanges over
// lane bits 4, 3, 2, 1 (6, 3, 2 and 1 shuffles; the 3 slots left after bit 3 are padded
// to 4) and a final add over bit 0, lane l holds in c[0] the warp sum of slot
// g + 3 b3 + 6 b4, g = (l >> 1) & 3, when l is even and g < 3. Returns that slot, or 12
// for the lanes that hold none.
__device__ __forceinline__ uint32_t warp_reduce_scatter12(float c[12], uint32_t lane) {
  const bool b4 = lane & 16u, b3 = lane & 8u, b2 = lane & 4u, b1 = lane & 2u;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const float send = b4 ? c[i] : c[i + 6];
    const float keep = b4 ? c[i + 6] : c[i];
    c[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float send = b3 ? c[i] : c[i + 3];
    const float keep = b3 ? c[i + 3] : c[i];
    c[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  {
    const float send0 = b2 ? c[0] : c[2];
    const float keep0 = b2 ? c[2] : c[0];
    const float send1 = b2 ? c[1] : 0.0f;
    const float keep1 = b2 ? 0.0f : c[1];
    c[0] = keep0 + __shfl_xor_sync(0xffffffffu, send0, 4);
    c[1] = keep1 + __shfl_xor_sync(0xffffffffu, send1, 4);
  }
  {
    const float send = b1 ? c[0] : c[1];
    const float keep = b1 ? c[1] : c[0];
    c[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  }
  c[0] += __shfl_xor_sync(0xffffffffu, c[0], 1);
  const uint32_t group = (lane >> 1) & 3u;
  return ((lane & 1u) == 0u && group < 3u) ? group + (b3 ? 3u : 0u) + (b4 ? 6u : 0u) : 12u;
}

// The fast mode's sum of a splat's 9 gradient values (without the |dmean| sums) over a
// warp's 32 lanes, through shared memory: each lane stores its values as a row of 12 floats
// (three conflict-free 16-byte stores); lane v + 9h (v < 9, h < 3) adds value v down the
// rows h, h + 3, h + 6, ... in two interleaved chains (the three groups' banks meet once)
// and returns that third of the sum (lanes 27-31 return 0). The warp sum of value v is
// third(v) + third(v + 9) + third(v + 18), in that order: warp_sum9_rows adds them with
// two shuffles; the split backward stores the thirds and lets one lane add them per round.
// Fewer instructions than a shuffle butterfly, which spends two selects per shuffle.
// `rows` is the warp's own 32 x 12 scratch.
__device__ __forceinline__ float warp_sum9_thirds(float (*rows)[12], const float c[12], uint32_t lane) {
  __syncwarp();  // the previous splat's rows have been read
  float4* row = reinterpret_cast<float4*>(&rows[lane][0]);
  row[0] = make_float4(c[0], c[1], c[2], c[3]);
  row[1] = make_float4(c[4], c[5], c[6], c[7]);
  row[2] = make_float4(c[8], 0.0f, 0.0f, 0.0f);
  __syncwarp();
  float even = 0.0f, odd = 0.0f;
  if (lane < 27u) {
    const uint32_t v = lane % 9u, h = lane / 9u;
#pragma unroll
    for (uint32_t i = 0; i < 10u; i += 2u) {
      even += rows[3u * i + h][v];
      odd += rows[3u * i + 3u + h][v];
    }
    if (30u + h < 32u) even += rows[30u + h][v];
  }
  return even + odd;
}

// The warp sum of value `lane` for lanes below 9 (warp_sum9_thirds).
__device__ __forceinline__ float warp_sum9_rows(float (*rows)[12], const float c[12], uint32_t lane) {
  const float sum = warp_sum9_thirds(rows, c, lane);
  return sum + __shfl_down_sync(0xffffffffu, sum, 9) + __shfl_down_sync(0xffffffffu, sum, 18);
}

// The tile and pixel layout of one block.
template <int PX>
struct TileLayout {
  static constexpr int kThreads = 256 / PX;
  static constexpr int kWarps = kThreads / 32;
  uint32_t v, t, W, H, tx, ty;
  float bx, by;  // centre of the warp block's first pixel
  __device__ TileLayout(const ViewTable* vt, const gs_frame_data* frames, uint32_t gt, uint32_t warp) {
    v = view_of_tile(vt, gt);
    const gs_frame_data& f = frames[v];
    W = f.image[0];
    H = f.image[1];
    t = gt - vt->tile_base[v];
    tx = t % f.image[2];
    ty = t / f.image[2];
    bx = float(tx * kTile + (warp & 1u) * 8u) + 0.5f;
    by = float(ty * kTile + (warp >> 1) * 4u * PX) + 0.5f;
  }
  // Pixel p of lane `lane`.
  __device__ uint2 pixel(uint32_t lane, int p) const {
    return make_uint2(uint32_t(bx - 0.5f) + (lane & 7u), uint32_t(by - 0.5f) + (lane >> 3) + 4u * uint32_t(p));
  }
};

// The next work item of a persistent block: tiles of the flattened (view, tile) space, in
// order, handed out by an atomic counter; `total` or more ends the loop.
__device__ __forceinline__ uint32_t next_tile(uint32_t* queue) {
  __shared__ uint32_t s_item;
  if (threadIdx.x == 0) s_item = atomicAdd(queue, 1u);
  __syncthreads();
  const uint32_t item = s_item;
  __syncthreads();
  return item;
}

// One staged splat blended into a warp's PX pixels at 1-based position `contributor` of the
// tile's list (train_forward.comp:96-121); returns whether all the lane's pixels are done.
template <int PX, bool COUNT>
__device__ __forceinline__ bool splat_blend(const float4 A, const float4 B, const float blue, const uint32_t contributor,
                                            const float cx, const float (&cy)[PX], bool (&done)[PX], float (&T)[PX],
                                            float (&C0)[PX], float (&C1)[PX], float (&C2)[PX], uint32_t (&last)[PX],
                                            uint32_t& blended) {
  const float dx = __fsub_rn(A.x, cx);
  const float e0 = __fmul_rn(__fmul_rn(A.w, dx), dx), e1 = __fmul_rn(B.x, dx);
  bool all_done = true;
#pragma unroll
  for (int p = 0; p < PX; ++p) {
    // Predicated rather than branched: a pixel that is done, or skips this splat, blends
    // it with alpha 0, which adds zero weight and keeps T (T (1 - 0) = T) and its last
    // contributor, bit for bit. Where it blends, T (1 - alpha) is the same product the
    // stop test formed.
    const float e = splat_exponent(e0, e1, B.y, __fsub_rn(A.y, cy[p]));
    const float alpha = fminf(kMaxAlpha, __fmul_rn(A.z, exp2_approx(e)));
    const bool blend = !done[p] && e <= 0.0f && alpha >= kMinAlpha;
    const bool stop = blend && __fmul_rn(T[p], __fsub_rn(1.0f, alpha)) < kMinTransmittance;
    const bool ok = blend && !stop;
    done[p] = done[p] || stop;
    const float ab = ok ? alpha : 0.0f;
    const float weight = ab * T[p];
    C0[p] += B.z * weight;
    C1[p] += B.w * weight;
    C2[p] += blue * weight;
    T[p] = __fmul_rn(T[p], __fsub_rn(1.0f, ab));
    last[p] = ok ? contributor : last[p];
    if constexpr (COUNT) blended += ok ? 1u : 0u;
    all_done = all_done && done[p];
  }
  return all_done;
}

// The forward's per-pixel outputs of a warp's PX pixels (train_forward.comp:123-183): colour over
// the background, dL/dC of the L1 part and final T, the last contributor, the RGBA8 image and
// dL/dC . C; and the warp's 14 loss and fit sums in vals (every lane holds the warp's total,
// summed by a butterfly in a fixed order). Returns the warp's furthest last contributor.
template <int PX>
__device__ __forceinline__ uint32_t pixels_out(const RasterArgs& a, const TileLayout<PX>& lay, const gs_frame_data& f,
                                               const uint32_t lane, const bool (&inside)[PX], const float cx,
                                               const float (&cy)[PX], const float (&T)[PX], const float (&C0)[PX],
                                               const float (&C1)[PX], const float (&C2)[PX],
                                               const uint32_t (&last)[PX], float (&vals)[14]) {
#pragma unroll
  for (int k = 0; k < 14; ++k) vals[k] = 0.0f;
  uint32_t my_max = 0u;
#pragma unroll
  for (int p = 0; p < PX; ++p) {
    if (!inside[p]) continue;
    const uint2 px = lay.pixel(lane, p);
    const size_t local = size_t(px.y) * lay.W + px.x;
    const size_t pix = size_t(a.vt->pixel_base[lay.v]) + local;
    const float o0 = C0[p] + T[p] * f.background[0], o1 = C1[p] + T[p] * f.background[1],
                o2 = C2[p] + T[p] * f.background[2];
    float d0 = 0.0f, d1 = 0.0f, d2 = 0.0f, w = 1.0f;
    const uint32_t* target = a.vt->target[lay.v];
    if (target != nullptr) {
      const uint32_t u = target[local];
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
      w = pixel_weight(make_float4(f.head[0], f.head[1], f.head[2], f.head[3]), cx, cy[p]);
      const float s = (1.0f - f.loss[0]) * f.background[3] * w;
      d0 = e0 > 0.0f ? s : (e0 < 0.0f ? -s : 0.0f);
      d1 = e1 > 0.0f ? s : (e1 < 0.0f ? -s : 0.0f);
      d2 = e2 > 0.0f ? s : (e2 < 0.0f ? -s : 0.0f);
      const float l0 = fabsf(e0) + fabsf(e1) + fabsf(e2);
      const float l1 = e0 * e0 + e1 * e1 + e2 * e2;
      vals[0] += l0;
      vals[1] += l1;
      vals[2] += w * l0;
      vals[3] += 3.0f * w;
      const float hx = cx - f.head[0], hy = cy[p] - f.head[1];
      if (f.head[2] > 0.0f && sqrtf(hx * hx + hy * hy) <= f.head[2]) {
        vals[4] += l1;
        vals[5] += 1.0f;
      }
      if (ta > 0.95f && T[p] < 0.05f) {
        vals[6] += C0[p] * C0[p];
        vals[7] += C1[p] * C1[p];
        vals[8] += C2[p] * C2[p];
        vals[9] += 1.0f;
        vals[10] += C0[p] * tr[0];
        vals[11] += C1[p] * tr[1];
        vals[12] += C2[p] * tr[2];
      }
      vals[13] += ta > 0.0f ? 1.0f : 0.0f;
    }
    a.rb.pixel_out[pix] = make_float4(o0, o1, o2, w);
    a.rb.pixel_grad[pix] = make_float4(d0, d1, d2, T[p]);
    a.rb.pixel_count[pix] = last[p];
    a.rb.image[pix] = pack_unorm(o0) | pack_unorm(o1) << 8 | pack_unorm(o2) << 16 | pack_unorm(1.0f - T[p]) << 24;
    a.rb.pixel_dot[pix] = d0 * o0 + d1 * o1 + d2 * o2;
    my_max = max(my_max, last[p]);
  }
  // The warp's sums, by a butterfly in a fixed order.
#pragma unroll
  for (int k = 0; k < 14; ++k) {
    float x = vals[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    vals[k] = x;
  }
  return __reduce_max_sync(0xffffffffu, my_max);
}

// COUNT: also add up the evaluations that blend (alpha >= 1/255, in front of the pixel's
// stop) into *contributions, for the work figure of the pass's roofline.
// FB splats are staged per round (64, 128 or 256: a tuning knob). With ASYNC the records of
// round i + 1 are copied with cp.async while round i blends (double-buffered raw records,
// the gaussian indices loaded one round further ahead), and each thread turns the records it
// copied into staged splats once they land.
template <int PX, int FB, bool ASYNC, bool COUNT>
__device__ __forceinline__ void raster_fwd_tile(const RasterArgs& a, uint32_t gt) {
  using L = TileLayout<PX>;
  static_assert(FB % 32 == 0 && FB <= 256, "whole warps of staged splats");
  constexpr int kPer = (FB + L::kThreads - 1) / L::kThreads;  // slots per thread
  __shared__ float4 s_a[FB];  // staged splats (stage_splat)
  __shared__ float4 s_b[FB];
  __shared__ float4 s_c[FB];
  __shared__ RawRound<ASYNC ? FB : 1> s_raw[ASYNC ? 2 : 1];
  __shared__ float s_red[L::kWarps][16];
  __shared__ uint32_t s_max[L::kWarps];

  const uint32_t lid = threadIdx.x, lane = lid & 31u, warp = lid >> 5;
  const L lay(a.vt, a.frames, gt, warp);
  const gs_frame_data& f = a.frames[lay.v];
  const uint2 range = a.rb.ranges[gt];

  bool inside[PX], done[PX];
  float cx = 0.0f, cy[PX], T[PX], C0[PX], C1[PX], C2[PX];
  uint32_t last[PX];
  uint32_t blended = 0u;  // COUNT
  bool all_done = true;
#pragma unroll
  for (int p = 0; p < PX; ++p) {
    const uint2 px = lay.pixel(lane, p);
    inside[p] = px.x < lay.W && px.y < lay.H;
    done[p] = !inside[p];
    all_done = all_done && done[p];
    cx = float(px.x) + 0.5f;
    cy[p] = float(px.y) + 0.5f;
    T[p] = 1.0f;
    C0[p] = C1[p] = C2[p] = 0.0f;
    last[p] = 0u;
  }
  const float block_h = float(4 * PX);
  uint32_t g_next[kPer];  // ASYNC: the gaussians of the round after the one in flight
  uint32_t buf = 0u;
  if constexpr (ASYNC) {
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
      const uint32_t slot = lid + uint32_t(r) * L::kThreads, k = range.x + slot;
      if (slot < uint32_t(FB) && k < range.y)
        fetch_record_async(&s_raw[0].q[0][slot], &s_raw[0].q[1][slot], &s_raw[0].q[2][slot], &s_raw[0].q[3][slot],
                           a.splat, a.foot, a.rb.gauss[k]);
    }
    copy_async_commit();
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
      const uint32_t slot = lid + uint32_t(r) * L::kThreads, k = range.x + uint32_t(FB) + slot;
      g_next[r] = slot < uint32_t(FB) && k < range.y ? a.rb.gauss[k] : 0u;
    }
  }
  for (uint32_t start = range.x; start < range.y; start += uint32_t(FB)) {
    if (__syncthreads_count(all_done) == L::kThreads) break;
    if constexpr (ASYNC) {
      // Round i + 1 into the other buffer (free: every warp has passed the barrier above),
      // then round i's own copies, staged by the thread that made them.
      const uint32_t nstart = start + uint32_t(FB);
#pragma unroll
      for (int r = 0; r < kPer; ++r) {
        const uint32_t slot = lid + uint32_t(r) * L::kThreads, k = nstart + slot;
        if (slot < uint32_t(FB) && k < range.y)
          fetch_record_async(&s_raw[buf ^ 1u].q[0][slot], &s_raw[buf ^ 1u].q[1][slot], &s_raw[buf ^ 1u].q[2][slot],
                             &s_raw[buf ^ 1u].q[3][slot], a.splat, a.foot, g_next[r]);
      }
      copy_async_commit();
#pragma unroll
      for (int r = 0; r < kPer; ++r) {
        const uint32_t slot = lid + uint32_t(r) * L::kThreads, k = nstart + uint32_t(FB) + slot;
        g_next[r] = slot < uint32_t(FB) && k < range.y ? a.rb.gauss[k] : 0u;
      }
      copy_async_wait<1>();
#pragma unroll
      for (int r = 0; r < kPer; ++r) {
        const uint32_t slot = lid + uint32_t(r) * L::kThreads;
        if (slot < uint32_t(FB) && start + slot < range.y) {
          float4 A, B, C;
          stage_splat(s_raw[buf].q[0][slot], s_raw[buf].q[1][slot], s_raw[buf].q[2][slot], s_raw[buf].q[3][slot].w,
                      A, B, C);
          s_a[slot] = A;
          s_b[slot] = B;
          s_c[slot] = C;
        }
      }
      buf ^= 1u;
    } else {
#pragma unroll
      for (uint32_t slot = lid; slot < uint32_t(FB); slot += uint32_t(L::kThreads)) {
        const uint32_t k = start + slot;
        if (k < range.y) {
          const uint32_t g = a.rb.gauss[k];
          const float4 q0 = a.splat[size_t(g) * 3u], q1 = a.splat[size_t(g) * 3u + 1u],
                       q2 = a.splat[size_t(g) * 3u + 2u];
          float4 A, B, C;
          stage_splat(q0, q1, q2, a.foot[g].w, A, B, C);
          s_a[slot] = A;
          s_b[slot] = B;
          s_c[slot] = C;
        }
      }
    }
    __syncthreads();
    const uint32_t n = min(uint32_t(FB), range.y - start);
    // The splats of this batch whose footprint reaches the warp's block, in order.
    uint32_t masks[FB / 32];
#pragma unroll
    for (int w = 0; w < FB / 32; ++w) {
      const uint32_t j = uint32_t(w) * 32u + lane;
      masks[w] = __ballot_sync(0xffffffffu, j < n && block_reached(s_a[j], s_b[j], s_c[j], lay.bx, lay.by, block_h));
    }
    const uint32_t base = start - range.x;  // position in the tile's list of the batch's first splat
#pragma unroll
    for (int w = 0; w < FB / 32; ++w) {
      uint32_t m = masks[w];
      while (m != 0u && !all_done) {
        const uint32_t j = uint32_t(w) * 32u + uint32_t(__ffs(m) - 1);
        m &= m - 1u;
        const uint32_t contributor = base + j + 1u;
        all_done = splat_blend<PX, COUNT>(s_a[j], s_b[j], s_c[j].x, contributor, cx, cy, done, T, C0, C1, C2, last,
                                          blended);
      }
    }
  }
  if constexpr (ASYNC) copy_async_wait<0>();  // no copy may land in the next tile's buffers

  float vals[14];
  const uint32_t wmax = pixels_out<PX>(a, lay, f, lane, inside, cx, cy, T, C0, C1, C2, last, vals);
  if constexpr (COUNT) {
    const uint32_t wsum = __reduce_add_sync(0xffffffffu, blended);
    if (lane == 0 && wsum) atomicAdd(a.contributions, static_cast<unsigned long long>(wsum));
  }
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 14; ++k) s_red[warp][k] = vals[k];
    s_max[warp] = wmax;
  }
  __syncthreads();
  if (lid < 16) {
    float s = 0.0f;
    if (lid < 14)
      for (int w8 = 0; w8 < L::kWarps; ++w8) s += s_red[w8][lid];
    // Layout of train_forward.comp:18-23 (slots 2 and 4 are the SSIM pass's):
    // values 0, 1 -> slots 0, 1; value 2 -> slot 3; values 3..13 -> slots 5..15.
    float* tl = a.rb.tile_loss + size_t(gt) * 16u;
    if (lid < 14) tl[lid < 2 ? lid : (lid == 2 ? 3 : lid + 2)] = s;
    if (lid == 14) tl[2] = 0.0f;
    if (lid == 15) tl[4] = 0.0f;
  }
  if (lid == 0) {
    uint32_t m = 0u;
    for (int w8 = 0; w8 < L::kWarps; ++w8) m = max(m, s_max[w8]);
    a.rb.tile_count[gt] = m;
  }
}

template <int PX, int FB, bool ASYNC, bool COUNT = false>
__global__ void __launch_bounds__(256 / PX) k_raster_fwd(RasterArgs a) {
  const uint32_t total = a.vt->total_tiles;
  for (uint32_t gt = next_tile(a.queue); gt < total; gt = next_tile(a.queue))
    raster_fwd_tile<PX, FB, ASYNC, COUNT>(a, gt);
}

// One staged splat's adjoint over a warp's PX row groups (train_common.glsl:215-253; the
// front-to-back form described at the top of the file), at 1-based position `pos` of the
// tile's list: updates each lane's T and R and, when some lane of the warp blends the
// splat, forms the splat's gradient values over the lane's pixels in c (11 with the
// |dmean| sums (ABS), else 9) and returns true. With RAW c holds the lane's sums before
// the splat's own factors instead, (u, dx u, dx^2 u, st, dx st, sty, the three colour
// weights, and with ABS the |dmean| sums without the opacity), linear in the lane's
// values, so the warp sums them first and raw_to_grads applies the opacity and the conic
// once per splat.
template <int PX, bool ABS, bool RAW = false>
__device__ __forceinline__ bool splat_adjoint(const float4 A, const float4 B, const float blue, const uint32_t pos,
                                              const float cx, const float (&cy)[PX], const float (&dl0)[PX],
                                              const float (&dl1)[PX], const float (&dl2)[PX],
                                              const uint32_t (&last)[PX], float (&T)[PX], float (&R)[PX],
                                              float (&c)[12]) {
  const float dx = __fsub_rn(A.x, cx);
  const float e0 = __fmul_rn(__fmul_rn(A.w, dx), dx), e1 = __fmul_rn(B.x, dx);
  // The conic (a, b, c) back from the scaled exponent terms, for the mean gradient:
  // dmx = dpow (lx + mx dy), dmy = dpow (ly + my dy).
  const float ca = A.w * (-2.0f / kLog2e), cb = B.x * (-1.0f / kLog2e), cc = B.y * (-2.0f / kLog2e);
  const float lx = -ca * dx, ly = -cb * dx, mx = -cb, my = -cc;
  // The lane's pixels share dx, so the mean and conic sums need only
  // sd = sum dpow, st = sum dpow dy and sty = sum dpow dy^2 (formed after the loop):
  // dmean = (lx sd + mx st, ly sd + my st), dconic = (-dx^2/2 sd, -dx st, -sty/2).
  // With dpow = opacity G dl the loop sums u = sum G dl (also the opacity gradient)
  // and st, sty over G dl; the opacity factor is applied once after it.
  float u = 0.0f, st = 0.0f, sty = 0.0f;
#pragma unroll
  for (int k = 6; k < 12; ++k) c[k] = 0.0f;
  // Whether some lane of the warp blends in some group. Without ABS it is set, warp-uniform,
  // by the groups' votes below; with ABS from each lane's tests and one more vote, which
  // measured faster in the deterministic kernel.
  bool has = false;
  float dy[PX], G[PX], raw[PX], alpha[PX];
  bool blend[PX];
#pragma unroll
  for (int p = 0; p < PX; ++p) {  // the groups' exponentials, independent of each other
    dy[p] = __fsub_rn(A.y, cy[p]);
    const float e = splat_exponent(e0, e1, B.y, dy[p]);
    G[p] = exp2_approx(e);
    raw[p] = __fmul_rn(A.z, G[p]);
    alpha[p] = fminf(kMaxAlpha, raw[p]);
    blend[p] = pos <= last[p] && e <= 0.0f && alpha[p] >= kMinAlpha;
    if constexpr (ABS) has = has || blend[p];
  }
  // Then the groups' adjoints, each skipped by the whole warp when no lane blends; a
  // lane that does not blend takes alpha 0, which leaves its T and R as they are and
  // adds nothing (its G dl is zeroed, so a G outside the footprint cannot make a NaN).
#pragma unroll
  for (int p = 0; p < PX; ++p) {
    if (!__any_sync(0xffffffffu, blend[p])) continue;
    if constexpr (!ABS) has = true;
    const float ab = blend[p] ? alpha[p] : 0.0f;
    const float gc = dl0[p] * B.z + dl1[p] * B.w + dl2[p] * blue;
    const float weight = ab * T[p];
    const float rest = R[p] - gc * weight;
    const float one_minus = __fsub_rn(1.0f, ab);
    const float dlda = T[p] * gc - __fdividef(rest, one_minus);
    // Opacity and exponent gradients vanish where alpha is clamped at 0.99.
    const float gd = (blend[p] && raw[p] < kMaxAlpha) ? G[p] * dlda : 0.0f;
    const float t = gd * dy[p];
    u += gd;
    st += t;
    sty = fmaf(t, dy[p], sty);
    c[6] += weight * dl0[p];
    c[7] += weight * dl1[p];
    c[8] += weight * dl2[p];
    if constexpr (ABS) {
      c[9] += fabsf(fmaf(t, mx, gd * lx));  // |dpow (lx + mx dy)| / opacity
      c[10] += fabsf(fmaf(t, my, gd * ly));
    }
    T[p] = __fmul_rn(T[p], one_minus);
    R[p] = rest;
  }
  if constexpr (ABS) has = __any_sync(0xffffffffu, has);
  if (!has) return false;
  if constexpr (RAW) {
    c[0] = u;
    c[1] = dx * u;
    c[2] = dx * c[1];
    c[3] = st;
    c[4] = dx * st;
    c[5] = sty;
    return true;
  }
  const float sd = A.z * u;
  st *= A.z;
  sty *= A.z;
  c[0] = fmaf(lx, sd, mx * st);
  c[1] = fmaf(ly, sd, my * st);
  c[2] = (-0.5f * dx * dx) * sd;
  c[3] = -dx * st;
  c[4] = -0.5f * sty;
  c[5] = u;
  if constexpr (ABS) {
    c[9] *= A.z;
    c[10] *= A.z;
  }
  return true;
}

// The splat's gradient values from the warp sums of splat_adjoint's raw terms r (in
// place): with op the opacity and the conic (ca, cb, cc) back from the staged exponent
// terms, dmean = -op (ca S(dx u) + cb S(st), cb S(dx u) + cc S(st)), dconic = -op
// (S(dx^2 u) / 2, S(dx st), S(sty) / 2), dopacity = S(u), |dmean| (ABS) = op S(|.|); the
// colour weights are unchanged.
template <bool ABS>
__device__ __forceinline__ void raw_to_grads(const float4 A, const float4 B, float (&r)[12]) {
  const float ca = A.w * (-2.0f / kLog2e), cb = B.x * (-1.0f / kLog2e), cc = B.y * (-2.0f / kLog2e);
  const float op = A.z;
  const float u = r[0], dxu = r[1], dx2u = r[2], st = r[3], dxst = r[4], sty = r[5];
  r[0] = -op * fmaf(ca, dxu, cb * st);
  r[1] = -op * fmaf(cb, dxu, cc * st);
  r[2] = (-0.5f * op) * dx2u;
  r[3] = -op * dxst;
  r[4] = (-0.5f * op) * sty;
  r[5] = u;
  if constexpr (ABS) {
    r[9] *= op;
    r[10] *= op;
  }
}

// The forward with independent warps (the default without stage_async). A work item is one
// warp's 8 x 4PX block of a tile (TileLayout<PX>); the warp stages its own rounds of 32
// splats from the tile's list and stops when all its pixels are done, with no block
// barrier. Each warp publishes its 14 tile sums and its furthest last contributor; the
// warp that finishes a tile last (a per-tile counter) adds the warps' sums in warp order,
// the same order as raster_fwd_tile, so the tile sums are bit-identical to it, writes
// them, and resets the counter for the next step.
struct FwdSplitSmem {
  float4 a[32], b[32], c[32];  // the round's staged splats (stage_splat)
};

template <int PX, bool COUNT>
__device__ __forceinline__ void raster_fwd_split(const RasterArgs& a, uint32_t item, uint32_t lane,
                                                 FwdSplitSmem& sm) {
  using L = TileLayout<PX>;
  const uint32_t gt = item / uint32_t(L::kWarps), warp = item - gt * uint32_t(L::kWarps);
  const L lay(a.vt, a.frames, gt, warp);
  const gs_frame_data& f = a.frames[lay.v];
  const uint2 range = a.rb.ranges[gt];

  bool inside[PX], done[PX];
  float cx = 0.0f, cy[PX], T[PX], C0[PX], C1[PX], C2[PX];
  uint32_t last[PX];
  uint32_t blended = 0u;  // COUNT
  bool all_done = true;
#pragma unroll
  for (int p = 0; p < PX; ++p) {
    const uint2 px = lay.pixel(lane, p);
    inside[p] = px.x < lay.W && px.y < lay.H;
    done[p] = !inside[p];
    all_done = all_done && done[p];
    cx = float(px.x) + 0.5f;
    cy[p] = float(px.y) + 0.5f;
    T[p] = 1.0f;
    C0[p] = C1[p] = C2[p] = 0.0f;
    last[p] = 0u;
  }
  const float block_h = float(4 * PX);
  for (uint32_t start = range.x; start < range.y; start += 32u) {
    if (__all_sync(0xffffffffu, all_done)) break;
    __syncwarp();  // the previous round's reads of the staging buffers are done
    const uint32_t k = start + lane;
    float4 A = make_float4(0.f, 0.f, 0.f, 0.f), B = A, C = A;
    if (k < range.y) {
      const uint32_t g = a.rb.gauss[k];
      const float4 q0 = a.splat[size_t(g) * 3u], q1 = a.splat[size_t(g) * 3u + 1u], q2 = a.splat[size_t(g) * 3u + 2u];
      stage_splat(q0, q1, q2, a.foot[g].w, A, B, C);
      sm.a[lane] = A;
      sm.b[lane] = B;
      sm.c[lane] = C;
    }
    __syncwarp();
    uint32_t m = __ballot_sync(0xffffffffu, k < range.y && block_reached(A, B, C, lay.bx, lay.by, block_h));
    const uint32_t base = start - range.x;  // position in the tile's list of the round's first splat
    while (m != 0u && !all_done) {
      const uint32_t j = uint32_t(__ffs(m) - 1);
      m &= m - 1u;
      all_done = splat_blend<PX, COUNT>(sm.a[j], sm.b[j], sm.c[j].x, base + j + 1u, cx, cy, done, T, C0, C1, C2, last,
                                        blended);
    }
  }

  float vals[14];
  const uint32_t wmax = pixels_out<PX>(a, lay, f, lane, inside, cx, cy, T, C0, C1, C2, last, vals);
  if constexpr (COUNT) {
    const uint32_t wsum = __reduce_add_sync(0xffffffffu, blended);
    if (lane == 0 && wsum) atomicAdd(a.contributions, static_cast<unsigned long long>(wsum));
  }
  float* parts = a.rb.tile_part + size_t(gt) * (kTileWarpSlots * 16u);
  uint32_t last_warp = 0u;
  if (lane == 0) {
#pragma unroll
    for (int v = 0; v < 14; ++v) parts[warp * 16u + uint32_t(v)] = vals[v];
    parts[warp * 16u + 14u] = __uint_as_float(wmax);
    __threadfence();  // the sums are visible before the count says so
    last_warp = atomicAdd(a.rb.tile_done + gt, 1u) == uint32_t(L::kWarps) - 1u ? 1u : 0u;
  }
  if (__shfl_sync(0xffffffffu, last_warp, 0) == 0u) return;
  __threadfence();
  if (lane < 16u) {
    float sum = 0.0f;
    if (lane < 14u)
      for (int w8 = 0; w8 < L::kWarps; ++w8) sum += __ldcg(parts + w8 * 16 + int(lane));
    // Layout of train_forward.comp:18-23 (slots 2 and 4 are the SSIM pass's):
    // values 0, 1 -> slots 0, 1; value 2 -> slot 3; values 3..13 -> slots 5..15.
    float* tl = a.rb.tile_loss + size_t(gt) * 16u;
    if (lane < 14u) tl[lane < 2u ? lane : (lane == 2u ? 3u : lane + 2u)] = sum;
    if (lane == 14u) tl[2] = 0.0f;
    if (lane == 15u) tl[4] = 0.0f;
  }
  if (lane == 0u) {
    uint32_t most = 0u;
    for (int w8 = 0; w8 < L::kWarps; ++w8) most = max(most, __float_as_uint(__ldcg(parts + w8 * 16 + 14)));
    a.rb.tile_count[gt] = most;
    a.rb.tile_done[gt] = 0u;
  }
}

// Four independent warps a block, each with its own staging buffers (8 blocks per SM; 6 at
// 4 pixels per thread, whose 64-register cap would spill).
template <int PX, bool COUNT>
__global__ void __launch_bounds__(128, PX == 4 ? 6 : 8) k_raster_fwd_split(RasterArgs a) {
  __shared__ __align__(16) FwdSplitSmem s_warp[4];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t total = a.vt->total_tiles * uint32_t(TileLayout<PX>::kWarps);
  for (;;) {
    uint32_t item = 0u;
    if (lane == 0u) item = atomicAdd(a.queue, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= total) break;
    raster_fwd_split<PX, COUNT>(a, item, lane, s_warp[warp]);
  }
}

// ASYNC: the splat records of round i + 1 are copied with cp.async while round i is
// differentiated (as in the forward).
template <int BATCH, int PX, bool ASYNC>
__device__ __forceinline__ void raster_bwd_tile(const RasterArgs& a, uint32_t gt) {
  constexpr bool DET = true;  // this layout serves the deterministic mode (fast mode: raster_bwd_split)
  constexpr bool ABS = DET;  // the |dL/dmean2d| sums (see the top of the file)
  using L = TileLayout<PX>;
  static_assert(BATCH <= L::kThreads, "one staged splat per thread");
  __shared__ float4 s_a[BATCH];
  __shared__ float4 s_b[BATCH];
  __shared__ float4 s_c[BATCH];  // staged splats (stage_splat): s_a, s_b, s_c
  __shared__ RawRound<ASYNC ? BATCH : 1> s_raw[ASYNC ? 2 : 1];
  __shared__ uint32_t s_dst[BATCH];
  __shared__ __align__(16) float s_part[L::kWarps][BATCH][12];
  __shared__ uint32_t s_wrote[L::kWarps][BATCH / 32];  // per warp: the splats whose partial it wrote

  const uint32_t lid = threadIdx.x, lane = lid & 31u, warp = lid >> 5;
  const L lay(a.vt, a.frames, gt, warp);
  const uint2 range = a.rb.ranges[gt];
  const uint32_t len = range.y - range.x;
  const uint32_t n = min(len, a.rb.tile_count[gt]);
  if (DET) {
    // Pairs behind the tile's furthest last contributor draw nothing (train_backward_serial.glsl:58-66).
    for (uint32_t k = range.x + n + lid; k < range.y; k += L::kThreads) {
      float4* o = reinterpret_cast<float4*>(a.pair_grads + size_t(a.rb.values[k]) * 12u);
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      o[0] = z;
      o[1] = z;
      o[2] = z;
    }
  }
  if (n == 0u) return;

  float cx = 0.0f, cy[PX], dl0[PX], dl1[PX], dl2[PX], R[PX], T[PX];
  uint32_t last[PX], my_last = 0u;
#pragma unroll
  for (int p = 0; p < PX; ++p) {
    const uint2 px = lay.pixel(lane, p);
    cx = float(px.x) + 0.5f;
    cy[p] = float(px.y) + 0.5f;
    dl0[p] = dl1[p] = dl2[p] = R[p] = 0.0f;
    T[p] = 1.0f;
    last[p] = 0u;
    if (px.x < lay.W && px.y < lay.H) {
      const size_t pix = size_t(a.vt->pixel_base[lay.v]) + size_t(px.y) * lay.W + px.x;
      const float4 pg = a.rb.pixel_grad[pix];
      dl0[p] = pg.x;
      dl1[p] = pg.y;
      dl2[p] = pg.z;
      R[p] = a.rb.pixel_dot[pix];
      last[p] = a.rb.pixel_count[pix];
      my_last = max(my_last, last[p]);
    }
  }
  const uint32_t wlast = __reduce_max_sync(0xffffffffu, my_last);
  const float block_h = float(4 * PX);

  // ASYNC: this thread's slot of the round in flight (cur) and of the next one (nxt): the
  // gaussian, and in deterministic mode the pair's pre-sort index (its gradient's place).
  const bool stager = lid < uint32_t(BATCH);
  uint32_t g_cur = 0u, pre_cur = 0u, g_nxt = 0u, pre_nxt = 0u, buf = 0u;
  if constexpr (ASYNC) {
    if (stager && lid < n) {
      g_cur = a.rb.gauss[range.x + lid];
      if (DET) pre_cur = a.rb.values[range.x + lid];
      fetch_record_async(&s_raw[0].q[0][lid], &s_raw[0].q[1][lid], &s_raw[0].q[2][lid], &s_raw[0].q[3][lid], a.splat,
                         a.foot, g_cur);
    }
    copy_async_commit();
    if (stager && uint32_t(BATCH) + lid < n) {
      g_nxt = a.rb.gauss[range.x + uint32_t(BATCH) + lid];
      if (DET) pre_nxt = a.rb.values[range.x + uint32_t(BATCH) + lid];
    }
  }
  for (uint32_t start = 0; start < n; start += BATCH) {
    __syncthreads();
    if constexpr (ASYNC) {
      // Round i + 1 into the other buffer (free: every warp has passed the barrier above),
      // the round after it's indices, then round i's own copy, staged by this thread.
      const bool next = stager && start + uint32_t(BATCH) + lid < n;
      if (next)
        fetch_record_async(&s_raw[buf ^ 1u].q[0][lid], &s_raw[buf ^ 1u].q[1][lid], &s_raw[buf ^ 1u].q[2][lid],
                           &s_raw[buf ^ 1u].q[3][lid], a.splat, a.foot, g_nxt);
      copy_async_commit();
      uint32_t g_after = 0u, pre_after = 0u;
      if (stager && start + 2u * uint32_t(BATCH) + lid < n) {
        g_after = a.rb.gauss[range.x + start + 2u * uint32_t(BATCH) + lid];
        if (DET) pre_after = a.rb.values[range.x + start + 2u * uint32_t(BATCH) + lid];
      }
      copy_async_wait<1>();
      if (stager && start + lid < n) {
        float4 A, B, C;
        stage_splat(s_raw[buf].q[0][lid], s_raw[buf].q[1][lid], s_raw[buf].q[2][lid], s_raw[buf].q[3][lid].w, A, B, C);
        s_a[lid] = A;
        s_b[lid] = B;
        s_c[lid] = C;
        s_dst[lid] = DET ? pre_cur : g_cur;
      }
      g_cur = g_nxt;
      pre_cur = pre_nxt;
      g_nxt = g_after;
      pre_nxt = pre_after;
      buf ^= 1u;
    } else if (stager && start + lid < n) {
      const uint32_t k = range.x + start + lid;
      const uint32_t g = a.rb.gauss[k];
      const float4 q0 = a.splat[size_t(g) * 3u], q1 = a.splat[size_t(g) * 3u + 1u], q2 = a.splat[size_t(g) * 3u + 2u];
      float4 A, B, C;
      stage_splat(q0, q1, q2, a.foot[g].w, A, B, C);
      s_a[lid] = A;
      s_b[lid] = B;
      s_c[lid] = C;
      s_dst[lid] = DET ? a.rb.values[k] : g;
    }
    __syncthreads();
    const uint32_t nb = min(uint32_t(BATCH), n - start);
    const uint32_t jmax = wlast > start ? min(nb, wlast - start) : 0u;
#pragma unroll
    for (int w = 0; w < BATCH / 32; ++w) {
      const uint32_t jj = uint32_t(w) * 32u + lane;
      uint32_t m = __ballot_sync(0xffffffffu, jj < jmax && block_reached(s_a[jj], s_b[jj], s_c[jj], lay.bx, lay.by, block_h));
      uint32_t wrote = 0u;
#pragma unroll 1
      while (m != 0u) {
        const uint32_t j = uint32_t(w) * 32u + uint32_t(__ffs(m) - 1);
        m &= m - 1u;
        const uint32_t pos = start + j + 1u;  // 1-based position in the tile's list
        float c[12];
        if (splat_adjoint<PX, ABS, true>(s_a[j], s_b[j], s_c[j].x, pos, cx, cy, dl0, dl1, dl2, last, T, R, c)) {
          const uint32_t slot = warp_reduce_scatter12(c, lane);
          if (slot < 12u) s_part[warp][j][slot] = c[0];
          wrote |= 1u << (j & 31u);
        }
      }
      if (lane == 0) s_wrote[warp][w] = wrote;
    }
    __syncthreads();
    // The pair's gradient at its pre-sort index: the warps' raw partials added in order,
    // then the splat's factors applied (zero for a splat no warp drew), for
    // train_pair_sum's fixed-order sum per gaussian.
    for (uint32_t j = lid; j < nb; j += L::kThreads) {
      float r[12];
#pragma unroll
      for (int k = 0; k < 12; ++k) r[k] = 0.0f;
      bool drawn = false;
#pragma unroll
      for (int w8 = 0; w8 < L::kWarps; ++w8) {
        if (((s_wrote[w8][j >> 5] >> (j & 31u)) & 1u) == 0u) continue;
        drawn = true;
        const float4* part = reinterpret_cast<const float4*>(&s_part[w8][j][0]);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const float4 v = part[q];
          r[4 * q] += v.x;
          r[4 * q + 1] += v.y;
          r[4 * q + 2] += v.z;
          r[4 * q + 3] += v.w;
        }
      }
      if (drawn) raw_to_grads<ABS>(s_a[j], s_b[j], r);
      float4* o = reinterpret_cast<float4*>(a.pair_grads + size_t(s_dst[j]) * 12u);
      o[0] = make_float4(r[0], r[1], r[2], r[3]);
      o[1] = make_float4(r[4], r[5], r[6], r[7]);
      o[2] = make_float4(r[8], r[9], r[10], r[11]);
    }
  }
  if constexpr (ASYNC) copy_async_wait<0>();  // no copy may land in the next tile's buffers
}

// One warp per 16x16 tile (backward_pixels = 8). Lane (c, r) = (lane & 7, lane >> 3) owns
// the tile's pixels (8h + c, 4q + r), p = 2q + h for h in {0, 1} and q in 0..3: the two
// half-tile warps of the 2-warp layout folded into one. Each warp takes tiles from the
// queue on its own and stages 32 splats per round, one per lane, with no block barrier. A
// splat reaching the tile is reduced once over the whole tile instead of once per half,
// and its sum needs no second, cross-warp stage. The lane's pixels share one of two dx
// values, so the mean and conic sums keep three per-lane sums per column half h:
// u = sum G dl (dpow = opacity G dl), s1 = sum G dl dy and s2 = sum G dl dy^2.
struct WarpTileSmem {
  float4 a[32], b[32], c[32];  // staged splats (stage_splat)
  uint32_t dst[32];            // pre-sort pair index (deterministic) or gaussian
  float part[32][12];          // the round's per-splat tile sums
  float lanes[32][12];         // the lanes' values of the splat being summed (fast mode)
};

template <bool DET>
__device__ __forceinline__ void raster_bwd_warp_tile(const RasterArgs& a, uint32_t gt, uint32_t lane,
                                                     WarpTileSmem& sm) {
  constexpr bool ABS = DET;  // the |dL/dmean2d| sums (see the top of the file)
  const uint32_t v = view_of_tile(a.vt, gt);
  const gs_frame_data& f = a.frames[v];
  const uint32_t W = f.image[0], H = f.image[1];
  const uint32_t t = gt - a.vt->tile_base[v];
  const uint32_t tx = t % f.image[2], ty = t / f.image[2];
  const uint2 range = a.rb.ranges[gt];
  const uint32_t len = range.y - range.x;
  const uint32_t n = min(len, a.rb.tile_count[gt]);
  if (DET) {
    // Pairs behind the tile's furthest last contributor draw nothing (train_backward_serial.glsl:58-66).
    for (uint32_t k = range.x + n + lane; k < range.y; k += 32u) {
      float4* o = reinterpret_cast<float4*>(a.pair_grads + size_t(a.rb.values[k]) * 12u);
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      o[0] = z;
      o[1] = z;
      o[2] = z;
    }
  }
  if (n == 0u) return;

  const uint32_t x0 = tx * kTile + (lane & 7u), y0 = ty * kTile + (lane >> 3);
  const float cx0 = float(x0) + 0.5f, cx1 = float(x0 + 8u) + 0.5f;
  float cy[4], dl0[8], dl1[8], dl2[8], R[8], T[8];
  uint32_t last[8], my_last = 0u;
#pragma unroll
  for (int q = 0; q < 4; ++q) cy[q] = float(y0 + 4u * uint32_t(q)) + 0.5f;
#pragma unroll
  for (int p = 0; p < 8; ++p) {
    const uint32_t x = x0 + 8u * uint32_t(p & 1), y = y0 + 4u * uint32_t(p >> 1);
    dl0[p] = dl1[p] = dl2[p] = R[p] = 0.0f;
    T[p] = 1.0f;
    last[p] = 0u;
    if (x < W && y < H) {
      const size_t pix = size_t(a.vt->pixel_base[v]) + size_t(y) * W + x;
      const float4 pg = a.rb.pixel_grad[pix];
      dl0[p] = pg.x;
      dl1[p] = pg.y;
      dl2[p] = pg.z;
      R[p] = a.rb.pixel_dot[pix];
      last[p] = a.rb.pixel_count[pix];
      my_last = max(my_last, last[p]);
    }
  }
  const uint32_t wlast = __reduce_max_sync(0xffffffffu, my_last);
  const float bx = float(tx * kTile) + 0.5f, by = float(ty * kTile) + 0.5f;

  for (uint32_t start = 0; start < n; start += 32u) {
    __syncwarp();  // the previous round's reads of the staging buffers are done
    float4 A = make_float4(0.f, 0.f, 0.f, 0.f), B = A, C = A;
    if (start + lane < n) {
      const uint32_t k = range.x + start + lane;
      const uint32_t g = a.rb.gauss[k];
      const float4 q0 = a.splat[size_t(g) * 3u], q1 = a.splat[size_t(g) * 3u + 1u], q2 = a.splat[size_t(g) * 3u + 2u];
      stage_splat(q0, q1, q2, a.foot[g].w, A, B, C);
      sm.a[lane] = A;
      sm.b[lane] = B;
      sm.c[lane] = C;
      sm.dst[lane] = DET ? a.rb.values[k] : g;
    }
    __syncwarp();
    const uint32_t nb = min(32u, n - start);
    const uint32_t jmax = wlast > start ? min(nb, wlast - start) : 0u;
    uint32_t m = __ballot_sync(0xffffffffu, lane < jmax && block_reached(A, B, C, bx, by, 16.0f, 16.0f));
    uint32_t wrote = 0u;
#pragma unroll 1
    while (m != 0u) {
      const uint32_t j = uint32_t(__ffs(m) - 1);
      m &= m - 1u;
      const uint32_t pos = start + j + 1u;  // 1-based position in the tile's list
      const float4 SA = sm.a[j];
      const float4 SB = sm.b[j];
      const float blue = sm.c[j].x;
      const float dx0 = __fsub_rn(SA.x, cx0), dx1 = __fsub_rn(SA.x, cx1);
      const float e00 = __fmul_rn(__fmul_rn(SA.w, dx0), dx0), e10 = __fmul_rn(SB.x, dx0);
      const float e01 = __fmul_rn(__fmul_rn(SA.w, dx1), dx1), e11 = __fmul_rn(SB.x, dx1);
      // The conic (a, b, c) back from the scaled exponent terms, for the mean gradient:
      // dmx = dpow (lx + mx dy), dmy = dpow (ly + my dy), lx = -ca dx, ly = -cb dx.
      const float ca = SA.w * (-2.0f / kLog2e), cb = SB.x * (-1.0f / kLog2e), cc = SB.y * (-2.0f / kLog2e);
      const float mx = -cb, my = -cc;
      float u[2] = {0.0f, 0.0f}, s1[2] = {0.0f, 0.0f}, s2[2] = {0.0f, 0.0f};
      float c[12];
#pragma unroll
      for (int k = 6; k < 12; ++k) c[k] = 0.0f;
      bool has = false;
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const int h = p & 1;
        if (pos > last[p]) continue;
        const float dy = __fsub_rn(SA.y, cy[p >> 1]);
        const float e = splat_exponent(h ? e01 : e00, h ? e11 : e10, SB.y, dy);
        const float G = exp2_approx(e);
        const float raw = __fmul_rn(SA.z, G);
        const float alpha = fminf(kMaxAlpha, raw);
        if (e > 0.0f || alpha < kMinAlpha) continue;
        has = true;
        const float gc = dl0[p] * SB.z + dl1[p] * SB.w + dl2[p] * blue;
        const float weight = alpha * T[p];
        const float rest = R[p] - gc * weight;
        const float one_minus = __fsub_rn(1.0f, alpha);
        const float dlda = T[p] * gc - __fdividef(rest, one_minus);
        // Opacity and exponent gradients vanish where alpha is clamped at 0.99.
        const float dl = raw >= kMaxAlpha ? 0.0f : dlda;
        const float gd = G * dl;  // dpow / opacity
        const float tt = gd * dy;
        u[h] += gd;
        s1[h] += tt;
        s2[h] = fmaf(tt, dy, s2[h]);
        c[6] += weight * dl0[p];
        c[7] += weight * dl1[p];
        c[8] += weight * dl2[p];
        if constexpr (ABS) {
          const float dx = h ? dx1 : dx0;
          c[9] += fabsf(fmaf(tt, mx, gd * (-ca * dx)));  // |dpow (lx + mx dy)| / opacity
          c[10] += fabsf(fmaf(tt, my, gd * (-cb * dx)));
        }
        T[p] = __fmul_rn(T[p], one_minus);
        R[p] = rest;
      }
      if (__any_sync(0xffffffffu, has)) {
        const float op = SA.z;
        const float sd0 = op * u[0], sd1 = op * u[1];
        const float sdx = fmaf(dx0, sd0, dx1 * sd1);                // sum dpow dx
        const float sdxx = fmaf(dx0 * dx0, sd0, (dx1 * dx1) * sd1);  // sum dpow dx^2
        const float st = op * (s1[0] + s1[1]);                      // sum dpow dy
        const float stx = op * fmaf(dx0, s1[0], dx1 * s1[1]);       // sum dpow dx dy
        const float sty = op * (s2[0] + s2[1]);                     // sum dpow dy^2
        c[0] = fmaf(-ca, sdx, mx * st);
        c[1] = fmaf(-cb, sdx, my * st);
        c[2] = -0.5f * sdxx;
        c[3] = -stx;
        c[4] = -0.5f * sty;
        c[5] = u[0] + u[1];
        if constexpr (ABS) {
          c[9] *= op;
          c[10] *= op;
        }
        if constexpr (ABS) {
          const uint32_t slot = warp_reduce_scatter12(c, lane);
          if (slot < 12u) sm.part[j][slot] = c[0];
        } else {
          const float sum = warp_sum9_rows(sm.lanes, c, lane);
          if (lane < 12u) sm.part[j][lane] = lane < 9u ? sum : 0.0f;
        }
        wrote |= 1u << j;
      }
    }
    __syncwarp();
    // Three float4s per staged splat: stored at the pair (deterministic; zero for a splat
    // that reached no pixel) or added to the gaussian's accumulator.
    for (uint32_t idx = lane; idx < nb * 3u; idx += 32u) {
      const uint32_t j = idx / 3u, qd = idx - 3u * j;
      const bool drew = (wrote >> j) & 1u;
      const float4 sum = drew ? *reinterpret_cast<const float4*>(&sm.part[j][4u * qd]) : make_float4(0.f, 0.f, 0.f, 0.f);
      if constexpr (DET) {
        reinterpret_cast<float4*>(a.pair_grads + size_t(sm.dst[j]) * 12u)[qd] = sum;
      } else if (drew) {
        atomicAdd(reinterpret_cast<float4*>(a.grad2d) + size_t(sm.dst[j]) * 3u + qd, sum);
      }
    }
  }
}

// Four independent warps per block, each with its own staging buffers; 5 blocks per SM
// (96 registers, no spills; a 6-block bound spills).
template <bool DET>
__global__ void __launch_bounds__(128, 5) k_raster_bwd_warp(RasterArgs a) {
  if (*a.d_pairs > a.accept) return;  // more pairs than stored: the step's update is skipped
  __shared__ WarpTileSmem s_warp[4];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t total = a.vt->total_tiles;
  for (;;) {
    uint32_t gt = 0u;
    if (lane == 0u) gt = atomicAdd(a.queue, 1u);
    gt = __shfl_sync(0xffffffffu, gt, 0);
    if (gt >= total) break;
    raster_bwd_warp_tile<DET>(a, gt, lane, s_warp[warp]);
  }
}

// Fast mode with independent warps. A work item is one warp's block of the tile layout of
// raster_bwd_tile (TileLayout<PX>: an 8 x 4PX block, 8 / PX of them a tile). The warp
// stages its own rounds of 32 splats from the tile's list, stops at its block's own
// furthest last contributor, and adds each splat's sums into the gaussian's accumulator
// with vector atomics, so no warp waits at a block barrier for another warp's pixels or
// round. Staging the tile's list once per warp instead of once per tile
// costs about 2% more instructions. (The deterministic mode adds the warps of a tile in a
// fixed order instead, in raster_bwd_tile.)
struct SplitSmem {
  float4 a[32], b[32], c[32];  // the round's staged splats (stage_splat)
  float part[32][28];          // the round's per-splat partial sums: value v of third h at v + 9h
  float lanes[32][12];         // the lanes' values of the splat being summed (warp_sum9_rows)
};

template <int PX>
__device__ __forceinline__ void raster_bwd_split(const RasterArgs& a, uint32_t item, uint32_t lane, SplitSmem& sm) {
  using L = TileLayout<PX>;
  const uint32_t gt = item / uint32_t(L::kWarps), warp = item - gt * uint32_t(L::kWarps);
  const L lay(a.vt, a.frames, gt, warp);
  const uint2 range = a.rb.ranges[gt];
  const uint32_t n = min(range.y - range.x, a.rb.tile_count[gt]);
  if (n == 0u) return;
  float cx = 0.0f, cy[PX], dl0[PX], dl1[PX], dl2[PX], R[PX], T[PX];
  uint32_t last[PX], my_last = 0u;
#pragma unroll
  for (int p = 0; p < PX; ++p) {
    const uint2 px = lay.pixel(lane, p);
    cx = float(px.x) + 0.5f;
    cy[p] = float(px.y) + 0.5f;
    dl0[p] = dl1[p] = dl2[p] = R[p] = 0.0f;
    T[p] = 1.0f;
    last[p] = 0u;
    if (px.x < lay.W && px.y < lay.H) {
      const size_t pix = size_t(a.vt->pixel_base[lay.v]) + size_t(px.y) * lay.W + px.x;
      const float4 pg = a.rb.pixel_grad[pix];
      dl0[p] = pg.x;
      dl1[p] = pg.y;
      dl2[p] = pg.z;
      R[p] = a.rb.pixel_dot[pix];
      last[p] = a.rb.pixel_count[pix];
      my_last = max(my_last, last[p]);
    }
  }
  const uint32_t stop = min(n, __reduce_max_sync(0xffffffffu, my_last));
  const float block_h = float(4 * PX);
  for (uint32_t start = 0; start < stop; start += 32u) {
    __syncwarp();  // the previous round's reads of the staging buffers are done
    float4 A = make_float4(0.f, 0.f, 0.f, 0.f), B = A, C = A;
    uint32_t g = 0u;  // the gaussian of the splat this lane stages
    if (start + lane < stop) {
      g = a.rb.gauss[range.x + start + lane];
      const float4 q0 = a.splat[size_t(g) * 3u], q1 = a.splat[size_t(g) * 3u + 1u], q2 = a.splat[size_t(g) * 3u + 2u];
      stage_splat(q0, q1, q2, a.foot[g].w, A, B, C);
      sm.a[lane] = A;
      sm.b[lane] = B;
      sm.c[lane] = C;
    }
    __syncwarp();
    const uint32_t nb = min(32u, stop - start);
    uint32_t m = __ballot_sync(0xffffffffu, lane < nb && block_reached(A, B, C, lay.bx, lay.by, block_h));
    uint32_t wrote = 0u;
#pragma unroll 1
    while (m != 0u) {
      const uint32_t j = uint32_t(__ffs(m) - 1);
      m &= m - 1u;
      float c[12];
      if (splat_adjoint<PX, false, true>(sm.a[j], sm.b[j], sm.c[j].x, start + j + 1u, cx, cy, dl0, dl1, dl2, last, T,
                                         R, c)) {
        const float third = warp_sum9_thirds(sm.lanes, c, lane);
        if (lane < 27u) sm.part[j][lane] = third;
        wrote |= 1u << j;
      }
    }
    __syncwarp();
    // Lane j staged splat j: it adds the three thirds of each warp sum, applies the splat's
    // factors (its own A and B) and adds the result into the gaussian's accumulator, two
    // 16-byte atomics and one for the ninth value.
    if ((wrote >> lane) & 1u) {
      const float4* row = reinterpret_cast<const float4*>(&sm.part[lane][0]);
      float t[28];
#pragma unroll
      for (int q = 0; q < 7; ++q) {
        const float4 x = row[q];
        t[4 * q] = x.x;
        t[4 * q + 1] = x.y;
        t[4 * q + 2] = x.z;
        t[4 * q + 3] = x.w;
      }
      float r[12];
#pragma unroll
      for (int v = 0; v < 9; ++v) r[v] = t[v] + t[v + 9] + t[v + 18];  // the thirds in lane order
      raw_to_grads<false>(A, B, r);
      float4* acc = reinterpret_cast<float4*>(a.grad2d) + size_t(g) * 3u;
      atomicAdd(acc, make_float4(r[0], r[1], r[2], r[3]));
      atomicAdd(acc + 1, make_float4(r[4], r[5], r[6], r[7]));
      atomicAdd(reinterpret_cast<float*>(acc + 2), r[8]);
    }
  }
}

// Four independent warps a block, each with its own staging buffers; 6 blocks per SM.
template <int PX>
__global__ void __launch_bounds__(128, 6) k_raster_bwd_split(RasterArgs a) {
  if (*a.d_pairs > a.accept) return;  // more pairs than stored: the step's update is skipped
  __shared__ __align__(16) SplitSmem s_warp[4];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t total = a.vt->total_tiles * uint32_t(TileLayout<PX>::kWarps);
  for (;;) {
    uint32_t item = 0u;
    if (lane == 0u) item = atomicAdd(a.queue, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= total) break;
    raster_bwd_split<PX>(a, item, lane, s_warp[warp]);
  }
}

// 3 PX blocks of 256 / PX threads per SM: 12 two-warp blocks at 4 pixels per thread (at
// most 85 registers; with no bound the compiler settled on 72 with spills, measured 1%
// slower, and a 64-register cap 18% slower).
template <int BATCH, int PX, bool ASYNC>
__global__ void __launch_bounds__(256 / PX, 3 * PX) k_raster_bwd(RasterArgs a) {
  if (*a.d_pairs > a.accept) return;  // more pairs than stored: the step's update is skipped
  const uint32_t total = a.vt->total_tiles;
  for (uint32_t gt = next_tile(a.queue); gt < total; gt = next_tile(a.queue))
    raster_bwd_tile<BATCH, PX, ASYNC>(a, gt);
}

// A persistent grid: as many blocks as fit on the GPU at once (at most one per tile).
template <typename Kernel>
uint32_t persistent_grid(Kernel kernel, int threads, const StepPointers& sp) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return min(sp.tile_cap, uint32_t(per_sm) * uint32_t(sp.sm_count));
}

template <int BATCH, int PX, bool ASYNC>
void launch_bwd(const RasterArgs& a, const StepPointers& sp, cudaStream_t st) {
  static uint32_t grid = 0, cap = 0;
  if (grid == 0 || cap != sp.tile_cap) {
    grid = persistent_grid(k_raster_bwd<BATCH, PX, ASYNC>, 256 / PX, sp);
    cap = sp.tile_cap;
  }
  k_raster_bwd<BATCH, PX, ASYNC><<<grid, 256 / PX, 0, st>>>(a);
}

template <bool DET>
void launch_bwd_warp(const RasterArgs& a, const StepPointers& sp, cudaStream_t st) {
  static uint32_t grid = 0, cap = 0;
  if (grid == 0 || cap != sp.tile_cap) {
    grid = persistent_grid(k_raster_bwd_warp<DET>, 128, sp);
    cap = sp.tile_cap;
  }
  k_raster_bwd_warp<DET><<<grid, 128, 0, st>>>(a);
}

template <int PX>
void launch_bwd_split(const RasterArgs& a, const StepPointers& sp, cudaStream_t st) {
  static uint32_t grid = 0, cap = 0;
  if (grid == 0 || cap != sp.tile_cap) {
    grid = persistent_grid(k_raster_bwd_split<PX>, 128, sp);
    cap = sp.tile_cap;
  }
  k_raster_bwd_split<PX><<<grid, 128, 0, st>>>(a);
}

// 8 pixels per thread: one warp per tile, either mode. Fast mode at 1, 2 or 4: the
// independent-warp kernel (its rounds are 32 splats and it stages with plain loads,
// whatever backward_batch and stage_async say). Deterministic mode at 1, 2 or 4: the
// block kernel, whose warps' partials are added in a fixed order.
template <int BATCH, bool DET, bool ASYNC>
void launch_bwd_px(const RasterArgs& a, const StepPointers& sp, int px, cudaStream_t st) {
  if (px >= 8) {
    launch_bwd_warp<DET>(a, sp, st);
  } else if constexpr (DET) {
    if (px >= 4) launch_bwd<BATCH, 4, ASYNC>(a, sp, st);
    else if (px == 2) launch_bwd<BATCH, 2, ASYNC>(a, sp, st);
    else launch_bwd<BATCH, 1, ASYNC>(a, sp, st);
  } else {
    if (px >= 4) launch_bwd_split<4>(a, sp, st);
    else if (px == 2) launch_bwd_split<2>(a, sp, st);
    else launch_bwd_split<1>(a, sp, st);
  }
}

template <int BATCH>
void launch_bwd_batch(const RasterArgs& a, const StepPointers& sp, bool deterministic, int px, bool async,
                      cudaStream_t st) {
  if (deterministic) {
    if (async) launch_bwd_px<BATCH, true, true>(a, sp, px, st);
    else launch_bwd_px<BATCH, true, false>(a, sp, px, st);
  } else {
    if (async) launch_bwd_px<BATCH, false, true>(a, sp, px, st);
    else launch_bwd_px<BATCH, false, false>(a, sp, px, st);
  }
}

template <int PX, int FB, bool ASYNC, bool COUNT = false>
void launch_fwd(const RasterArgs& a, const StepPointers& sp, cudaStream_t st) {
  static uint32_t grid = 0, cap = 0;
  if (grid == 0 || cap != sp.tile_cap) {
    grid = persistent_grid(k_raster_fwd<PX, FB, ASYNC, COUNT>, 256 / PX, sp);
    cap = sp.tile_cap;
  }
  k_raster_fwd<PX, FB, ASYNC, COUNT><<<grid, 256 / PX, 0, st>>>(a);
}

template <int PX, bool COUNT>
void launch_fwd_split(const RasterArgs& a, const StepPointers& sp, cudaStream_t st) {
  static uint32_t grid = 0, cap = 0;
  if (grid == 0 || cap != sp.tile_cap) {
    grid = persistent_grid(k_raster_fwd_split<PX, COUNT>, 128, sp);
    cap = sp.tile_cap;
  }
  k_raster_fwd_split<PX, COUNT><<<grid, 128, 0, st>>>(a);
}

template <int PX, bool ASYNC>
void launch_fwd_batch(const RasterArgs& a, const StepPointers& sp, int batch, cudaStream_t st) {
  if (batch >= 256) launch_fwd<PX, 256, ASYNC>(a, sp, st);
  else if (batch >= 128) launch_fwd<PX, 128, ASYNC>(a, sp, st);
  else launch_fwd<PX, 64, ASYNC>(a, sp, st);
}

template <int PX>
void launch_fwd_mode(const RasterArgs& a, const StepPointers& sp, int batch, bool async, cudaStream_t st) {
  if (async) launch_fwd_batch<PX, true>(a, sp, batch, st);
  else launch_fwd_batch<PX, false>(a, sp, batch, st);
}

}  // namespace

void launch_raster_forward(const StepPointers& sp, const ViewBuffers& vb, const RasterBuffers& rb, int px, int batch,
                           bool async, unsigned long long* contributions, cudaStream_t st) {
  if (sp.tile_cap == 0u) return;
  RasterArgs a{sp.frames, sp.vt, sp.queue + kQueueForward, rb, vb.splat, vb.foot, nullptr, nullptr, nullptr, 0u,
               contributions};
  if (contributions != nullptr) {  // the counting variant: same blend, plus the count
    if (px >= 4) launch_fwd_split<4, true>(a, sp, st);
    else if (px == 2) launch_fwd_split<2, true>(a, sp, st);
    else launch_fwd_split<1, true>(a, sp, st);
    return;
  }
  if (!async) {  // independent warps (their rounds are 32 splats whatever `batch` says)
    if (px >= 4) launch_fwd_split<4, false>(a, sp, st);
    else if (px == 2) launch_fwd_split<2, false>(a, sp, st);
    else launch_fwd_split<1, false>(a, sp, st);
    return;
  }
  if (px >= 4) launch_fwd_mode<4>(a, sp, batch, async, st);
  else if (px == 2) launch_fwd_mode<2>(a, sp, batch, async, st);
  else launch_fwd_mode<1>(a, sp, batch, async, st);
}

void launch_raster_backward(const StepPointers& sp, const ViewBuffers& vb, const RasterBuffers& rb,
                            float4* pair_grads, bool deterministic, int px, int batch, bool async,
                            const uint32_t* d_pairs, uint32_t accept, cudaStream_t st) {
  if (sp.tile_cap == 0u) return;
  RasterArgs a{sp.frames, sp.vt, sp.queue + kQueueBackward, rb, vb.splat, vb.foot,
               reinterpret_cast<float*>(pair_grads), reinterpret_cast<float*>(vb.grad2d), d_pairs, accept, nullptr};
  if (batch >= 64) launch_bwd_batch<64>(a, sp, deterministic, px, async, st);
  else launch_bwd_batch<32>(a, sp, deterministic, px, async, st);
}

}  // namespace gsk
