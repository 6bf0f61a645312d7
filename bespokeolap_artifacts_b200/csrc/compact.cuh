// Order-preserving stream compaction over an index range [0, n): the indices
// a predicate keeps, with one 32-bit value each, written in ascending index
// order (no atomics decide positions).  Three launches:
//   ordered_count_kernel  per tile of kCompactTile indices, the kept count;
//   ordered_scan_kernel   one block: exclusive scan of the tile counts, the
//                         total into *n_out;
//   ordered_emit_kernel   each tile again: per-thread counts, a block scan,
//                         and the kept values at tile offset + thread offset.
// A thread owns kCompactPerThread consecutive indices of its tile, so the
// output order is the index order.  The predicate is a device functor:
//   bool operator()(int64_t i, uint32_t& value) const.
// Used where a sort only existed to restore an index order (the TPC-H result
// rows whose ties keep ascending key order).
#pragma once

#include "common.cuh"
#include "context.cuh"

namespace bo {

constexpr int kCompactBlockT = 256;
constexpr int kCompactPerThread = 16;
constexpr int64_t kCompactTile = (int64_t)kCompactBlockT * kCompactPerThread;
constexpr int kCompactScanBlock = 1024;

// Exclusive block scan of one value per thread (blockDim.x == kCompactBlockT);
// returns the thread's offset, *total the block's sum.
__device__ __forceinline__ uint32_t compact_block_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t warp_tot[kCompactBlockT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  uint32_t before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kCompactBlockT / 32; ++w) {
    const uint32_t t = warp_tot[w];
    before += w < warp ? t : 0u;
    all += t;
  }
  __syncthreads();  // warp_tot may be reused by the caller's next scan
  *total = all;
  return before + x - v;
}

template <class Pred>
__global__ void __launch_bounds__(kCompactBlockT) ordered_count_kernel(Pred pred, int64_t n,
                                                                       uint32_t* __restrict__ tile_counts) {
  const int64_t t0 = (int64_t)blockIdx.x * kCompactTile + (int64_t)threadIdx.x * kCompactPerThread;
  uint32_t c = 0;
#pragma unroll
  for (int k = 0; k < kCompactPerThread; ++k) {
    uint32_t v;
    if (t0 + k < n && pred(t0 + k, v)) ++c;
  }
  uint32_t total;
  compact_block_scan(c, &total);
  if (threadIdx.x == 0) tile_counts[blockIdx.x] = total;
}

// In place: tile_counts[t] becomes the exclusive prefix; *n_out the total.
static __global__ void __launch_bounds__(kCompactScanBlock) ordered_scan_kernel(uint32_t* __restrict__ tile_counts,
                                                                         int64_t tiles,
                                                                         unsigned long long* __restrict__ n_out) {
  __shared__ unsigned long long warp_tot[kCompactScanBlock / 32];
  __shared__ unsigned long long carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < tiles; base += kCompactScanBlock) {
    const int64_t i = base + threadIdx.x;
    const unsigned long long v = i < tiles ? tile_counts[i] : 0ull;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    unsigned long long before = 0, all = 0;
    for (int w = 0; w < kCompactScanBlock / 32; ++w) {
      before += w < warp ? warp_tot[w] : 0ull;
      all += warp_tot[w];
    }
    const unsigned long long c = carry;
    if (i < tiles) tile_counts[i] = (uint32_t)(c + before + x - v);  // < 2^32: callers keep n below that
    __syncthreads();
    if (threadIdx.x == 0) carry = c + all;
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_out = carry;
}

template <class Pred>
__global__ void __launch_bounds__(kCompactBlockT) ordered_emit_kernel(Pred pred, int64_t n,
                                                                      const uint32_t* __restrict__ tile_offsets,
                                                                      uint32_t* __restrict__ out) {
  const int64_t t0 = (int64_t)blockIdx.x * kCompactTile + (int64_t)threadIdx.x * kCompactPerThread;
  uint32_t vals[kCompactPerThread];
  uint32_t keep = 0;
#pragma unroll
  for (int k = 0; k < kCompactPerThread; ++k) {
    vals[k] = 0;
    if (t0 + k < n && pred(t0 + k, vals[k])) keep |= 1u << k;
  }
  uint32_t total;
  uint32_t pos = tile_offsets[blockIdx.x] + compact_block_scan(__popc(keep), &total);
#pragma unroll
  for (int k = 0; k < kCompactPerThread; ++k)
    if ((keep >> k) & 1u) out[pos++] = vals[k];
}

// The three launches on the context's stream; tile_counts holds
// ceil(n / kCompactTile) words.  Returns a status (launch errors).
template <class Pred>
int ordered_compact(bo_ctx* ctx, const Pred& pred, int64_t n, uint32_t* tile_counts, uint32_t* out,
                    unsigned long long* n_out) {
  const int64_t tiles = (n + kCompactTile - 1) / kCompactTile;
  if (tiles == 0) {
    BO_CUDA(ctx, cudaMemsetAsync(n_out, 0, sizeof(unsigned long long), ctx->stream));
    return BO_OK;
  }
  if (n > 0xffffffffll) return set_error(ctx, BO_ERR_INVALID, "ordered_compact: %lld indices", (long long)n);
  ordered_count_kernel<Pred><<<(unsigned)tiles, kCompactBlockT, 0, ctx->stream>>>(pred, n, tile_counts);
  int rc = after_launch(ctx, "ordered_count_kernel");
  if (rc) return rc;
  ordered_scan_kernel<<<1, kCompactScanBlock, 0, ctx->stream>>>(tile_counts, tiles, n_out);
  if ((rc = after_launch(ctx, "ordered_scan_kernel"))) return rc;
  ordered_emit_kernel<Pred><<<(unsigned)tiles, kCompactBlockT, 0, ctx->stream>>>(pred, n, tile_counts, out);
  return after_launch(ctx, "ordered_emit_kernel");
}

// Order-preserving compaction of a bitmap: the positions of the set bits of
// words[0 .. n_words), ascending, into out; their number into *n_out.  Same
// three launches, a thread owning kBitmapWordsPerThread consecutive words
// (a tile covers kCompactBlockT * kBitmapWordsPerThread * 32 positions), so
// the passes read the bitmap, not a per-position predicate's inputs.
constexpr int kBitmapWordsPerThread = 4;
constexpr int64_t kBitmapTileWords = (int64_t)kCompactBlockT * kBitmapWordsPerThread;

static __global__ void __launch_bounds__(kCompactBlockT) bitmap_count_kernel(const uint32_t* __restrict__ words,
                                                                            int64_t n_words,
                                                                            uint32_t* __restrict__ tile_counts) {
  const int64_t w0 = (int64_t)blockIdx.x * kBitmapTileWords + (int64_t)threadIdx.x * kBitmapWordsPerThread;
  uint32_t c = 0;
#pragma unroll
  for (int k = 0; k < kBitmapWordsPerThread; ++k)
    if (w0 + k < n_words) c += __popc(__ldg(words + w0 + k));
  uint32_t total;
  compact_block_scan(c, &total);
  if (threadIdx.x == 0) tile_counts[blockIdx.x] = total;
}

static __global__ void __launch_bounds__(kCompactBlockT) bitmap_emit_kernel(const uint32_t* __restrict__ words,
                                                                           int64_t n_words,
                                                                           const uint32_t* __restrict__ tile_offsets,
                                                                           uint32_t* __restrict__ out) {
  const int64_t w0 = (int64_t)blockIdx.x * kBitmapTileWords + (int64_t)threadIdx.x * kBitmapWordsPerThread;
  uint32_t w[kBitmapWordsPerThread];
  uint32_t c = 0;
#pragma unroll
  for (int k = 0; k < kBitmapWordsPerThread; ++k) {
    w[k] = w0 + k < n_words ? __ldg(words + w0 + k) : 0u;
    c += __popc(w[k]);
  }
  uint32_t total;
  uint32_t pos = tile_offsets[blockIdx.x] + compact_block_scan(c, &total);
#pragma unroll
  for (int k = 0; k < kBitmapWordsPerThread; ++k) {
    uint32_t x = w[k];
    while (x) {
      const int b = __ffs(x) - 1;
      out[pos++] = (uint32_t)((w0 + k) * 32 + b);
      x &= x - 1u;
    }
  }
}

// tile_counts holds ceil(n_words / kBitmapTileWords) words; positions must
// be below 2^32.
inline int bitmap_compact(bo_ctx* ctx, const uint32_t* words, int64_t n_words, uint32_t* tile_counts, uint32_t* out,
                          unsigned long long* n_out) {
  const int64_t tiles = (n_words + kBitmapTileWords - 1) / kBitmapTileWords;
  if (tiles == 0) {
    BO_CUDA(ctx, cudaMemsetAsync(n_out, 0, sizeof(unsigned long long), ctx->stream));
    return BO_OK;
  }
  if (n_words > (int64_t)(0xffffffffll / 32)) return set_error(ctx, BO_ERR_INVALID, "bitmap_compact: %lld words", (long long)n_words);
  bitmap_count_kernel<<<(unsigned)tiles, kCompactBlockT, 0, ctx->stream>>>(words, n_words, tile_counts);
  int rc = after_launch(ctx, "bitmap_count_kernel");
  if (rc) return rc;
  ordered_scan_kernel<<<1, kCompactScanBlock, 0, ctx->stream>>>(tile_counts, tiles, n_out);
  if ((rc = after_launch(ctx, "ordered_scan_kernel"))) return rc;
  bitmap_emit_kernel<<<(unsigned)tiles, kCompactBlockT, 0, ctx->stream>>>(words, n_words, tile_counts, out);
  return after_launch(ctx, "bitmap_emit_kernel");
}

}  // namespace bo
