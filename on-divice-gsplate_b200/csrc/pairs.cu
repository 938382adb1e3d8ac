// Pair emission and tile ranges.
//
// launch_emit: train_emit.comp:26-64. Items come in depth order (the depth sort of every
// (view, slot)); each writes its (tile, gaussian) pairs at its scanned offset, over the
// same footprint rows train_project counted (train_common.glsl:185-213): the row spans the
// projection packed while counting, or, for footprints too large to pack, the same walk
// again from the stored records. The pair key is the global tile (view tile base + tile), so one stable
// sort by key leaves every tile's pairs front to back, ties in slot order — the order a
// (tile, depth16, index) sort gives (test_trainer.cpp:197-233).
// launch_ranges: train_ranges.comp:14-29 over the sorted keys.
#include "gs_kernels.h"

namespace gsk {
namespace {

struct EmitArgs {
  const gs_frame_data* frames;
  const ViewTable* vt;
  uint32_t cap, n_items, pair_capacity;
  const uint32_t* sorted_vals;
  const uint32_t* sorted_offsets;
  const uint32_t* total;  // the scan's total: the end of the last item's pairs
  const float4* splat;
  const float4* foot;
  const uint4* spans;
  uint32_t* offsets;  // first pair per g; null in atomic training steps (only snapshots read it)
  uint32_t* keys;
  uint32_t* values;
  uint32_t* pair_gaussian;  // g per pre-sort pair; null when the values carry g (nothing reads it then)
  float4* pair_grads;
  uint32_t* mismatch;
  bool payload_gaussian;  // values carry g instead of the pre-sort index
};

// Pairs a warp stages in shared memory before writing them out: a warp's items are
// consecutive in depth order, so their pairs form one contiguous range, written with
// coalesced stores instead of one scattered run per lane.
constexpr uint32_t kEmitStage = 512;

__global__ void __launch_bounds__(128) k_emit(EmitArgs a) {
  __shared__ uint32_t s_tile[4][kEmitStage];
  __shared__ uint32_t s_owner[4][kEmitStage];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (blockIdx.x * blockDim.x + warp * 32u >= a.n_items) return;  // the whole warp
  // The item's pairs [p, p + count) from consecutive scan offsets (coalesced): items that
  // emit nothing (the invisible ones, sorted last) need no gather.
  uint32_t p = 0u, count = 0u;
  if (k < a.n_items) {
    p = a.sorted_offsets[k];
    count = (k + 1u < a.n_items ? a.sorted_offsets[k + 1u] : *a.total) - p;
  }
  const uint32_t wfirst = __shfl_sync(0xffffffffu, p, 0);
  const uint32_t wend = min(__reduce_max_sync(0xffffffffu, count ? p + count : 0u), a.pair_capacity);
  if (wend <= wfirst) {
    if (count != 0u && a.offsets != nullptr) a.offsets[a.sorted_vals[k]] = p;  // all past the capacity
    return;
  }
  const bool staged = wend - wfirst <= kEmitStage;
  uint32_t* st_tile = s_tile[warp];
  uint32_t* st_owner = s_owner[warp];
  if (count != 0u) {
    const uint32_t g = a.sorted_vals[k];
    const uint32_t v = g / a.cap;
    const gs_frame_data& f = a.frames[v];
    const uint4 packed = a.spans[g];
    if (a.offsets != nullptr) a.offsets[g] = p;
    const uint32_t end = min(p + count, a.pair_capacity);
    const uint32_t tile_base = a.vt->tile_base[v];
    const uint32_t width = f.image[0], height = f.image[1], tiles_x = f.image[2];
    auto put = [&](uint32_t q, uint32_t tile) {
      if (staged) {
        st_tile[q - wfirst] = tile;
        st_owner[q - wfirst] = g;
      } else {
        a.keys[q] = tile;
        a.values[q] = a.payload_gaussian ? g : q;
        if (a.pair_gaussian != nullptr) a.pair_gaussian[q] = g;
      }
    };
    uint32_t wanted = 0u;
    if (packed.x >> 31) {
      // The row spans the projection packed while counting (footprint_count_spans).
      const uint32_t ty0 = packed.x & 0xffffu, n_rows = (packed.x >> 16) & 0xffu;
      const unsigned long long lo = packed.y | static_cast<unsigned long long>(packed.z) << 32;
      for (uint32_t r = 0; r < n_rows; ++r) {
        const uint32_t bits = r < 4u ? uint32_t(lo >> (16u * r)) & 0xffffu : (packed.w >> (16u * (r - 4u))) & 0xffffu;
        const uint32_t x0 = bits & 1023u, x1 = x0 + (bits >> 10);
        wanted += x1 - x0;
        const uint32_t row = tile_base + (ty0 + r) * tiles_x;
        for (uint32_t x = x0; x < x1 && p < end; ++x) put(p++, row + x);
      }
    } else {
      const float4 q0 = a.splat[size_t(g) * 3u];
      const float4 fp = a.foot[g];
      const int2 rows = footprint_rows(q0.x, q0.y, fp.z, fp.w, height);
      if (rows.x <= rows.y) {
        for (uint32_t ty = uint32_t(rows.x) / kTile; ty <= uint32_t(rows.y) / kTile; ++ty) {
          const uint2 span = footprint_row_tiles(q0.x, q0.y, fp.x, fp.y, fp.z, fp.w, rows, ty, width);
          wanted += span.y - span.x;
          for (uint32_t x = span.x; x < span.y && p < end; ++x) put(p++, tile_base + ty * tiles_x + x);
        }
      }
    }
    if (wanted != count) {
      // The count and the walk disagree (never expected: same inputs, same arithmetic).
      // Pad the rest into the unused tile after the last one, with zero gradient.
      atomicAdd(a.mismatch, 1u);
      const uint32_t pad_tile = a.vt->total_tiles;
      for (; p < end; ++p) {
        put(p, pad_tile);
        if (a.pair_grads != nullptr) {
          const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
          a.pair_grads[size_t(p) * 3u] = z;
          a.pair_grads[size_t(p) * 3u + 1u] = z;
          a.pair_grads[size_t(p) * 3u + 2u] = z;
        }
      }
    }
  }
  if (!staged) return;
  __syncwarp();
  for (uint32_t q = wfirst + lane; q < wend; q += 32u) {
    const uint32_t owner = st_owner[q - wfirst];
    a.keys[q] = st_tile[q - wfirst];
    a.values[q] = a.payload_gaussian ? owner : q;
    if (a.pair_gaussian != nullptr) a.pair_gaussian[q] = owner;
  }
}

// Grid-stride over the stored pairs, four consecutive keys per thread from one 16-byte
// load (the grid is sized for the SMs, not the capacity). At each tile boundary that is
// also a view boundary the view spans are written too.
__device__ __forceinline__ void range_edge(uint32_t s, uint32_t prev, uint32_t tile, uint2* ranges, const ViewTable* vt,
                                           uint32_t* view_span) {
  ranges[prev].y = s;
  ranges[tile].x = s;
  const uint32_t v = view_of_tile(vt, tile), vp = view_of_tile(vt, prev);
  if (v != vp) {
    view_span[v] = s;
    view_span[kMaxViews + vp] = s;
  }
}

__global__ void __launch_bounds__(256) k_ranges(const uint32_t* __restrict__ keys, const uint32_t* d_count,
                                                uint32_t capacity, uint2* __restrict__ ranges, const ViewTable* vt,
                                                uint32_t* __restrict__ view_span, PairGather gather) {
  const uint32_t count = min(*d_count, capacity);
  if (count == 0u) return;
  const uint32_t groups = (count + 3u) / 4u;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < groups; q += gridDim.x * blockDim.x) {
    const uint32_t s0 = 4u * q;
    uint32_t k[4];
    if (s0 + 4u <= count) {
      const uint4 v = *reinterpret_cast<const uint4*>(keys + s0);
      k[0] = v.x;
      k[1] = v.y;
      k[2] = v.z;
      k[3] = v.w;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) k[j] = s0 + j < count ? keys[s0 + j] : 0u;
    }
    if (gather.sorted_g != nullptr) {
      if (s0 + 4u <= count) {
        const uint4 v = *reinterpret_cast<const uint4*>(gather.sorted_values + s0);
        *reinterpret_cast<uint4*>(gather.sorted_g + s0) =
            make_uint4(gather.pair_gaussian[v.x], gather.pair_gaussian[v.y], gather.pair_gaussian[v.z],
                       gather.pair_gaussian[v.w]);
      } else {
        for (uint32_t s = s0; s < count; ++s) gather.sorted_g[s] = gather.pair_gaussian[gather.sorted_values[s]];
      }
    }
    uint32_t prev = s0 > 0u ? keys[s0 - 1u] : 0u;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t s = s0 + uint32_t(j);
      if (s >= count) break;
      const uint32_t tile = k[j];
      if (s == 0u) {
        ranges[tile].x = 0u;
        view_span[view_of_tile(vt, tile)] = 0u;
      } else if (prev != tile) {
        range_edge(s, prev, tile, ranges, vt, view_span);
      }
      if (s == count - 1u) {
        ranges[tile].y = count;
        view_span[kMaxViews + view_of_tile(vt, tile)] = count;
      }
      prev = tile;
    }
  }
}

}  // namespace

void launch_emit(const StepPointers& sp, const ViewBuffers& vb, uint32_t cap, uint32_t n_items,
                 const uint32_t* sorted_vals, const uint32_t* sorted_offsets, const uint32_t* total,
                 uint32_t pair_capacity, uint32_t* keys, uint32_t* values, uint32_t* pair_gaussian, float4* pair_grads,
                 uint32_t* mismatch, bool payload_gaussian, cudaStream_t st) {
  if (n_items == 0u) return;
  // An atomic training step (the gaussian as the payload) writes no first-pair offsets.
  uint32_t* offsets = payload_gaussian ? nullptr : vb.offsets;
  EmitArgs a{sp.frames, sp.vt,    cap,        n_items,  pair_capacity, sorted_vals, sorted_offsets,
             total,     vb.splat, vb.foot,    vb.spans, offsets,       keys,        values,
             pair_gaussian, pair_grads, mismatch, payload_gaussian};
  k_emit<<<(n_items + 127u) / 128u, 128, 0, st>>>(a);
}

void launch_ranges(const uint32_t* sorted_keys, const uint32_t* d_count, uint32_t pair_capacity, uint2* ranges,
                   const ViewTable* vt, uint32_t* view_span, const PairGather* gather, cudaStream_t st) {
  if (pair_capacity == 0u) return;
  k_ranges<<<min((pair_capacity + 1023u) / 1024u, 148u * 8u), 256, 0, st>>>(
      sorted_keys, d_count, pair_capacity, ranges, vt, view_span, gather ? *gather : PairGather{});
}

}  // namespace gsk
