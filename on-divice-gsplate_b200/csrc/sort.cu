// Device radix sort and exclusive scan.
//
// The reference sorts with a 3-kernel LSD radix sort of 4-bit digits (count, single
// workgroup scan, scatter: engine/src/radix_sort.cpp:57-108, radix_{count,scan,scatter}.comp)
// and scans with scan_local/blocks/add. Here:
//  - radix_sort_pairs: LSD sort, digits of 4 to 8 bits (8 by default; the width is a tuning
//    knob), three kernels a pass. k_tile_counts counts the digits of every 3840-key tile;
//    k_tile_scan turns each digit's row of tile counts into the tiles' starts within the
//    digit and the digit's total (one block per digit); k_rank_scatter ranks and scatters: a
//    block adds the totals of the smaller digits (one scan) to its tiles' starts, ranks its
//    tile's keys (same-digit lanes from one ballot per digit bit, per-warp counters,
//    stable) and writes each digit run contiguously through shared memory. The ballots
//    replace __match_any_sync, whose pipe was measured 87% busy with 8-bit digits (up to 32
//    distinct values per warp). No block waits on another: a decoupled look-back over the
//    previous tiles' counts was measured slower here, its polls of the same few status
//    lines serialising in L2. So this is a reduce-then-scan sort, not a single-pass
//    (onesweep) one: the look-back was built, measured and dropped.
//  - exclusive_scan: three kernels (tile sums with the gathered values staged in the
//    output, one block scanning the tile sums, then each tile's own scan), again with no
//    block waiting on another, so no kernel of the sort or the scan spins on a flag.
#include "gs_kernels.h"

namespace gsk {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kIpt = 15;  // keys per thread
constexpr int kRadix = 256;  // digit tables are sized for 8-bit digits; narrower digits use a prefix
__device__ __forceinline__ uint32_t count_of(const uint32_t* d_count, uint32_t n_max) {
  return d_count != nullptr ? min(*d_count, n_max) : n_max;
}

// Exclusive scan of one value per thread over a 256-thread block; returns the block total.
template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* s_warp, T& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  T warp_prefix = 0, sum = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    const T t = s_warp[w];
    if (w < warp) warp_prefix += t;
    sum += t;
  }
  __syncthreads();
  total = sum;
  return warp_prefix + x - v;
}

// Per-tile digit counts of one pass, digit-major: counts[d * stride + tile].
__global__ void __launch_bounds__(kThreads) k_tile_counts(const uint32_t* __restrict__ keys, const uint32_t* d_count,
                                                          uint32_t n_max, int shift, uint32_t mask,
                                                          uint32_t* __restrict__ counts, uint32_t stride) {
  __shared__ uint32_t s_count[kRadix];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t tile = blockIdx.x;
  const uint32_t n = count_of(d_count, n_max);
  const uint32_t base = tile * kSortTile;
  if (base >= n) return;
  s_count[tid] = 0u;
  __syncthreads();
  const uint32_t wbase = base + uint32_t(warp) * 32u * kIpt;
  uint32_t key[kIpt];
#pragma unroll
  for (int j = 0; j < kIpt; ++j) {
    const uint32_t idx = wbase + uint32_t(j) * 32u + lane;
    key[j] = idx < n ? keys[idx] : 0u;
  }
#pragma unroll
  for (int j = 0; j < kIpt; ++j) {
    const uint32_t idx = wbase + uint32_t(j) * 32u + lane;
    if (idx < n) atomicAdd(&s_count[(key[j] >> shift) & mask], 1u);
  }
  __syncthreads();
  counts[size_t(tid) * stride + tile] = s_count[tid];
}

// Digit `blockIdx.x`: its counts over the live tiles become each tile's start within the
// digit (the counts of the tiles before it, in place), and the digit's total goes to
// totals[d]. One 1024-thread block per digit: a row of up to 9216 tiles in one sweep.
constexpr int kRowThreads = 1024;
constexpr int kRowIpt = 9;
__global__ void __launch_bounds__(kRowThreads) k_tile_scan(uint32_t* __restrict__ counts, uint32_t stride,
                                                           const uint32_t* d_count, uint32_t n_max,
                                                           uint32_t* __restrict__ totals) {
  __shared__ uint32_t s_warp[kRowThreads / 32];
  __shared__ uint32_t s_carry;
  const uint32_t n = count_of(d_count, n_max);
  const uint32_t live = (n + kSortTile - 1u) / kSortTile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t* row = counts + size_t(blockIdx.x) * stride;
  uint32_t carry = 0u;
  for (uint32_t chunk = 0; chunk < live; chunk += kRowThreads * kRowIpt) {
    uint32_t x[kRowIpt], sum = 0u;
#pragma unroll
    for (int k = 0; k < kRowIpt; ++k) {
      const uint32_t t = chunk + uint32_t(threadIdx.x) * kRowIpt + k;
      x[k] = t < live ? row[t] : 0u;
      sum += x[k];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const uint32_t w = s_warp[lane];
      uint32_t wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += y;
      }
      s_warp[lane] = wi - w;  // exclusive prefix of the warps
    }
    __syncthreads();
    uint32_t run = carry + s_warp[warp] + incl - sum;
#pragma unroll
    for (int k = 0; k < kRowIpt; ++k) {
      const uint32_t t = chunk + uint32_t(threadIdx.x) * kRowIpt + k;
      if (t < live) row[t] = run;
      run += x[k];
    }
    if (threadIdx.x == kRowThreads - 1) s_carry = run;  // the last thread ends the chunk
    __syncthreads();
    carry = s_carry;
  }
  if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// Ranks of a warp's keys within its digit runs (stable), counting into the warp's row of
// s_wc. kFull: every key of the tile is valid (all tiles but the last), so no lane test.
template <bool kFull>
__device__ __forceinline__ void rank_keys(const uint32_t (&key)[kIpt], uint16_t (&rank)[kIpt], uint32_t* wc,
                                          uint32_t lane, uint32_t wbase, uint32_t n, int shift, uint32_t mask) {
  const uint32_t lanemask_lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < kIpt; ++j) {
    const bool valid = kFull || wbase + uint32_t(j) * 32u + lane < n;
    const uint32_t digit = valid ? (key[j] >> shift) & mask : uint32_t(kRadix);
    // The lanes holding the same digit, from one ballot per digit bit.
    uint32_t peers = kFull ? 0xffffffffu : __ballot_sync(0xffffffffu, valid);
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const bool bit = (digit >> b) & 1u;
      const uint32_t set = __ballot_sync(0xffffffffu, bit);
      peers &= bit ? set : ~set;
    }
    uint32_t before = 0u;
    if (valid) before = wc[digit];
    __syncwarp();
    if (valid && lane == uint32_t(__ffs(peers) - 1)) wc[digit] = before + __popc(peers);
    __syncwarp();
    rank[j] = uint16_t(before + __popc(peers & lanemask_lt));
  }
}

// One pass: each block ranks its tile's keys (same-digit lanes from ballots, per-warp
// counters, stable) and scatters them through shared memory to its digits' global starts.
__global__ void __launch_bounds__(kThreads, 4) k_rank_scatter(const uint32_t* __restrict__ keys_in,
                                                       const uint32_t* __restrict__ vals_in,
                                                       uint32_t* __restrict__ keys_out,
                                                       uint32_t* __restrict__ vals_out, const uint32_t* d_count,
                                                       uint32_t n_max, int shift, uint32_t mask,
                                                       const uint32_t* __restrict__ starts, uint32_t stride,
                                                       const uint32_t* __restrict__ totals) {
  __shared__ uint32_t s_wc[kWarps][kRadix];  // per-warp digit counts, then each warp's first block position per digit
  __shared__ uint32_t s_delta[kRadix];       // global position minus block position, per digit
  __shared__ unsigned long long s_warp[kWarps];
  __shared__ uint32_t s_keys[kSortTile];
  __shared__ uint32_t s_vals[kSortTile];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t tile = blockIdx.x;
  const uint32_t n = count_of(d_count, n_max);
  const uint32_t base = tile * kSortTile;
  if (base >= n) return;
  for (int k = tid; k < kWarps * kRadix; k += kThreads) (&s_wc[0][0])[k] = 0u;
  __syncthreads();

  uint32_t key[kIpt], val[kIpt];
  uint16_t rank[kIpt];
  const uint32_t wbase = base + uint32_t(warp) * 32u * kIpt;
#pragma unroll
  for (int j = 0; j < kIpt; ++j) {
    const uint32_t idx = wbase + uint32_t(j) * 32u + lane;
    if (idx < n) {
      key[j] = keys_in[idx];
      val[j] = vals_in[idx];
    } else {
      key[j] = 0xffffffffu;
      val[j] = 0u;
    }
  }
  if (base + kSortTile <= n) rank_keys<true>(key, rank, s_wc[warp], lane, wbase, n, shift, mask);
  else rank_keys<false>(key, rank, s_wc[warp], lane, wbase, n, shift, mask);
  __syncthreads();

  // Digit `tid`: block count and block-local start, then each warp's first block position
  // (one shared read per key in the scatter below). The digit's global start is the totals
  // of the smaller digits (one scan over the block, packed with the block's own counts)
  // plus the counts of the earlier tiles.
  const uint32_t start = starts[size_t(tid) * stride + tile];
  const uint32_t total = uint32_t(tid) <= mask ? totals[tid] : 0u;
  uint32_t count = 0u;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) count += s_wc[w][tid];
  unsigned long long both_total;
  const unsigned long long both =
      block_exclusive_scan<unsigned long long>((static_cast<unsigned long long>(total) << 32) | count, s_warp,
                                               both_total);
  const uint32_t dstart = uint32_t(both), digit_base = uint32_t(both >> 32);
  {
    uint32_t running = dstart;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t c = s_wc[w][tid];
      s_wc[w][tid] = running;
      running += c;
    }
  }
  s_delta[tid] = digit_base + start - dstart;
  if (tid == 0) s_warp[0] = static_cast<unsigned long long>(n) << 32 | uint32_t(shift);
  __syncthreads();
  // The shift and count read back from shared memory keep the scatter's digit and bounds
  // arithmetic below the barrier (computed earlier, they would hold registers through the
  // scan).
  const uint32_t shift2 = uint32_t(s_warp[0]), n2 = uint32_t(s_warp[0] >> 32);

#pragma unroll
  for (int j = 0; j < kIpt; ++j) {
    const uint32_t idx = wbase + uint32_t(j) * 32u + lane;
    if (idx < n2) {
      const uint32_t pos = s_wc[warp][(key[j] >> shift2) & mask] + rank[j];
      s_keys[pos] = key[j];
      s_vals[pos] = val[j];
    }
  }
  __syncthreads();
  const uint32_t tile_n = min(kSortTile, n - base);
  for (uint32_t p = tid; p < tile_n; p += kThreads) {
    const uint32_t k = s_keys[p];
    const uint32_t out = s_delta[(k >> shift) & mask] + p;
    keys_out[out] = k;
    vals_out[out] = s_vals[p];
  }
}

constexpr int kScanIpt = 8;

// Exclusive scan in three kernels, none waiting on another. k_scan_sums: each 2048-item
// tile gathers its values (through `gather` when given) into out[] and writes its sum;
// k_scan_tiles: one block turns the tile sums into tile starts (64-bit) and the total;
// k_scan_apply: each tile scans its gathered values from out[] and adds its start.
__global__ void __launch_bounds__(kThreads) k_scan_sums(const uint32_t* __restrict__ in,
                                                        const uint32_t* __restrict__ gather, uint32_t* __restrict__ out,
                                                        uint32_t n, unsigned long long* __restrict__ tile_sums) {
  __shared__ uint32_t s_warp[kWarps];
  const uint32_t base = blockIdx.x * kScanTile;
  uint32_t sum = 0u;
#pragma unroll
  for (int j = 0; j < kScanIpt; ++j) {
    const uint32_t idx = base + uint32_t(j) * kThreads + threadIdx.x;  // coalesced
    if (idx < n) {
      const uint32_t x = in[gather != nullptr ? gather[idx] : idx];
      out[idx] = x;
      sum += x;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if ((threadIdx.x & 31u) == 0u) s_warp[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < kWarps; ++w) t += s_warp[w];
    tile_sums[blockIdx.x] = t;
  }
}

constexpr int kTileScanThreads = 1024;
constexpr int kTileScanIpt = 4;

__global__ void __launch_bounds__(kTileScanThreads) k_scan_tiles(unsigned long long* __restrict__ tile_sums,
                                                                 uint32_t tiles, uint32_t* d_total) {
  __shared__ unsigned long long s_warp[kTileScanThreads / 32];
  __shared__ unsigned long long s_carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long carry = 0;
  for (uint32_t chunk = 0; chunk < tiles; chunk += kTileScanThreads * kTileScanIpt) {
    unsigned long long x[kTileScanIpt], sum = 0;
#pragma unroll
    for (int k = 0; k < kTileScanIpt; ++k) {
      const uint32_t t = chunk + uint32_t(threadIdx.x) * kTileScanIpt + k;
      x[k] = t < tiles ? tile_sums[t] : 0ull;
      sum += x[k];
    }
    unsigned long long incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const unsigned long long w = s_warp[lane];
      unsigned long long wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += y;
      }
      s_warp[lane] = wi - w;
    }
    __syncthreads();
    unsigned long long run = carry + s_warp[warp] + incl - sum;
#pragma unroll
    for (int k = 0; k < kTileScanIpt; ++k) {
      const uint32_t t = chunk + uint32_t(threadIdx.x) * kTileScanIpt + k;
      if (t < tiles) tile_sums[t] = run;
      run += x[k];
    }
    if (threadIdx.x == kTileScanThreads - 1) s_carry = run;
    __syncthreads();
    carry = s_carry;
  }
  if (threadIdx.x == 0 && d_total != nullptr) *d_total = uint32_t(carry);
}

__global__ void __launch_bounds__(kThreads) k_scan_apply(uint32_t* __restrict__ out, uint32_t n,
                                                         const unsigned long long* __restrict__ tile_starts) {
  __shared__ unsigned long long s_warp[kWarps];
  const uint32_t base = blockIdx.x * kScanTile;
  uint32_t x[kScanIpt];
  unsigned long long sum = 0;
#pragma unroll
  for (int j = 0; j < kScanIpt; ++j) {
    const uint32_t idx = base + uint32_t(threadIdx.x) * kScanIpt + j;
    x[j] = idx < n ? out[idx] : 0u;
    sum += x[j];
  }
  unsigned long long block_total;
  unsigned long long run =
      tile_starts[blockIdx.x] + block_exclusive_scan<unsigned long long>(sum, s_warp, block_total);
#pragma unroll
  for (int j = 0; j < kScanIpt; ++j) {
    const uint32_t idx = base + uint32_t(threadIdx.x) * kScanIpt + j;
    if (idx < n) out[idx] = uint32_t(run);
    run += x[j];
  }
}

}  // namespace

bool radix_sort_pairs(const SortScratch& s, uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt,
                      const uint32_t* d_count, uint32_t n_max, int bits, cudaStream_t st, int* launches,
                      int digit_bits) {
  if (n_max <= 1u || bits <= 0) return false;
  digit_bits = digit_bits < 4 ? 4 : (digit_bits > 8 ? 8 : digit_bits);
  const int passes = (bits + digit_bits - 1) / digit_bits;
  const uint32_t tiles = (n_max + kSortTile - 1u) / kSortTile;
  if (launches) *launches += 3 * passes;
  uint32_t *src_k = keys, *src_v = vals, *dst_k = keys_alt, *dst_v = vals_alt;
  for (int p = 0; p < passes; ++p) {
    const int shift = digit_bits * p;
    const int width = min(digit_bits, bits - shift);
    const uint32_t mask = (1u << width) - 1u;
    k_tile_counts<<<tiles, kThreads, 0, st>>>(src_k, d_count, n_max, shift, mask, s.tile_counts, tiles);
    k_tile_scan<<<mask + 1u, kRowThreads, 0, st>>>(s.tile_counts, tiles, d_count, n_max, s.hist + p * kRadix);
    k_rank_scatter<<<tiles, kThreads, 0, st>>>(src_k, src_v, dst_k, dst_v, d_count, n_max, shift, mask, s.tile_counts,
                                           tiles, s.hist + p * kRadix);
    uint32_t* t = src_k;
    src_k = dst_k;
    dst_k = t;
    t = src_v;
    src_v = dst_v;
    dst_v = t;
  }
  return (passes & 1) != 0;
}

void exclusive_scan(const SortScratch& s, const uint32_t* in, const uint32_t* gather, uint32_t* out, uint32_t n,
                    uint32_t* d_total, cudaStream_t st, int* launches) {
  if (n == 0u) {
    if (d_total) cudaMemsetAsync(d_total, 0, sizeof(uint32_t), st);
    return;
  }
  const uint32_t tiles = (n + kScanTile - 1u) / kScanTile;
  k_scan_sums<<<tiles, kThreads, 0, st>>>(in, gather, out, n, s.scan_lookback);
  k_scan_tiles<<<1, kTileScanThreads, 0, st>>>(s.scan_lookback, tiles, d_total);
  k_scan_apply<<<tiles, kThreads, 0, st>>>(out, n, s.scan_lookback);
  if (launches) *launches += 3;
}

}  // namespace gsk
