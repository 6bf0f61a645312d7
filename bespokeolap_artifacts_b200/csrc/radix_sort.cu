// LSD onesweep radix sort of (uint64 key, uint32 value) pairs with decoupled
// look-back (K5), and top-k as sort + truncate (K6).
//
// Reference counterpart: the stable LSD counting sorts with 16-bit digits of
// bespoke_tpch/query_q10.cpp:134-168, 285-316, 318-372 (descending order via
// ~key, ties kept in the order of the earlier passes), and the final ORDER BY
// std::sort calls (query_q3.cpp:348-355, query_q18.cpp:443-452,
// bespoke_ceb/query_q3b.cpp:1369-1385).
//
// Design (8-bit digits, only the passes covering [begin_bit, end_bit)):
//  * radix_hist_kernel -- one read of the keys builds every pass's 256-bin
//    histogram (shared-memory counters, one global atomic per bin per block);
//    its last block turns them into exclusive digit bases;
//  * radix_pass_kernel -- persistent blocks (at most the resident grid) take
//    tiles of 4096 keys in order from an atomic counter, so every predecessor
//    tile belongs to a running block.  A warp ranks its 512 keys
//    stably in 16 rounds of 32 (match_any on the digit, per-warp digit counters
//    in shared memory), the block sums its warps into tile counts, publishes
//    them, and each of the 256 threads does the decoupled look-back for one
//    digit over predecessor tiles' 64-bit status words
//    (flag:2 | epoch:30 | count:32), 16 predecessors per round trip.  The epoch (unique per pass launch) makes
//    stale words from earlier passes read as "not ready", so status arrays are
//    never cleared.  Every spin is bounded by the global timer; a timeout sets
//    an error bit instead of hanging.
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "context.cuh"

namespace bo {

constexpr int kSortBlock = 256;
constexpr int kSortWarps = kSortBlock / 32;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortBlock * kSortRounds;  // 4096 keys
constexpr int kRadix = 256;
constexpr int kMaxPasses = 8;
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagPrefix = 2ull << 62;

__device__ __forceinline__ int64_t sort_n(int64_t n, const unsigned long long* n_dev) {
  if (!n_dev) return n;
  const unsigned long long v = *n_dev;
  return v < (unsigned long long)n ? (int64_t)v : n;
}

// Histograms of every pass; the last block to finish turns them into
// exclusive digit bases in place (no separate scan launch).
__global__ void __launch_bounds__(kSortBlock) radix_hist_kernel(const unsigned long long* __restrict__ keys, int64_t n_max,
                                                                const unsigned long long* __restrict__ n_dev,
                                                                int begin_bit, int n_passes,
                                                                unsigned long long* __restrict__ hist,
                                                                uint32_t* __restrict__ done) {
  const int64_t n = sort_n(n_max, n_dev);
  if (n == 0) return;  // nothing to sort: no histogram, no ticket
  // Blocks past the actual count (the grid covers the upper bound) retire at
  // once; the last-block ticket counts only the blocks that hold keys.
  const int64_t blocks_needed = (n + blockDim.x - 1) / blockDim.x;
  const uint32_t active = blocks_needed < (int64_t)gridDim.x ? (uint32_t)blocks_needed : gridDim.x;
  if (blockIdx.x >= active) return;
  __shared__ uint32_t h[kMaxPasses][kRadix];
  for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += blockDim.x) (&h[0][0])[i] = 0;
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long k = keys[i];
    for (int p = 0; p < n_passes; ++p) atomicAdd(&h[p][(k >> (begin_bit + 8 * p)) & 0xffu], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n_passes * kRadix; i += blockDim.x)
    if ((&h[0][0])[i]) atomicAdd(&hist[i], (unsigned long long)(&h[0][0])[i]);
  if (!last_block(done, active)) return;
  __shared__ unsigned long long sc[kRadix];
  for (int p = 0; p < n_passes; ++p) {
    const unsigned long long v = __ldcg(&hist[p * kRadix + threadIdx.x]);
    sc[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kRadix; o <<= 1) {
      const unsigned long long add = threadIdx.x >= o ? sc[threadIdx.x - o] : 0ull;
      __syncthreads();
      sc[threadIdx.x] += add;
      __syncthreads();
    }
    hist[p * kRadix + threadIdx.x] = sc[threadIdx.x] - v;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kSortBlock) radix_pass_kernel(
    const unsigned long long* __restrict__ kin, const uint32_t* __restrict__ vin, unsigned long long* __restrict__ kout,
    uint32_t* __restrict__ vout, int64_t n_max, const unsigned long long* __restrict__ n_dev, int shift,
    const unsigned long long* __restrict__ digit_base, unsigned long long* status, uint32_t* tile_counter,
    uint32_t epoch, uint32_t* err) {
  // With the key count on the device, the grid covers the upper bound and the
  // tiles past the actual count retire at once (tile ids are handed out in
  // order, so no live tile ever looks back at them).
  const int64_t n = sort_n(n_max, n_dev);
  if (n == 0) return;  // nothing to sort: retire before touching the tile counter
  // Blocks beyond the tiles the actual count needs retire without a ticket
  // (block 0 always stays, and the staying blocks take every tile in order).
  if ((int64_t)blockIdx.x * kSortTile >= n) return;
  // A pass over a digit that every key shares (one non-empty bin) is the
  // identity permutation: the tiles are copied in place of ranking and
  // look-back.  Result sets of a few thousand keys sorted by 64-bit keys
  // have several such passes (complemented or narrow fields).
  {
    const unsigned long long lo = digit_base[threadIdx.x];
    const unsigned long long hi = threadIdx.x + 1 < kRadix ? digit_base[threadIdx.x + 1] : (unsigned long long)n;
    if (__syncthreads_count(hi > lo) == 1) {
      for (int64_t t = blockIdx.x; t * kSortTile < n; t += gridDim.x) {
        const int64_t end = min((t + 1) * (int64_t)kSortTile, n);
        for (int64_t i = t * kSortTile + threadIdx.x; i < end; i += kSortBlock) {
          kout[i] = kin[i];
          vout[i] = vin[i];
        }
      }
      return;
    }
  }
  __shared__ uint32_t warp_cnt[kSortWarps][kRadix];
  __shared__ unsigned long long tile_base[kRadix];
  __shared__ uint32_t tile_s;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt_mask = (1u << lane) - 1u;
  // Persistent blocks take tiles in order from the counter until the keys run
  // out (the grid is at most the resident grid, so every tile a block waits
  // on belongs to a running block that has already published its counts).
  for (;;) {
    for (int i = threadIdx.x; i < kSortWarps * kRadix; i += blockDim.x) (&warp_cnt[0][0])[i] = 0;
    if (threadIdx.x == 0) tile_s = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = tile_s;
    if ((int64_t)tile * kSortTile >= n) break;
    const int64_t seg = (int64_t)tile * kSortTile + (int64_t)warp * (32 * kSortRounds);

    unsigned long long key[kSortRounds];
    uint32_t val[kSortRounds];
    uint32_t rank[kSortRounds];
    uint32_t dig[kSortRounds];
    // Stable per-warp ranking: rounds in input order, lanes in input order.
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
      const int64_t idx = seg + r * 32 + lane;
      const bool valid = idx < n;
      key[r] = valid ? kin[idx] : 0ull;
      val[r] = valid ? vin[idx] : 0u;
      const uint32_t d = valid ? (uint32_t)((key[r] >> shift) & 0xffu) : 0x100u;
      dig[r] = d;
      const uint32_t peers = __match_any_sync(0xffffffffu, d);
      const uint32_t before = valid ? warp_cnt[warp][d] : 0u;
      __syncwarp();
      if (valid && lane == __ffs(peers) - 1) warp_cnt[warp][d] = before + __popc(peers);
      __syncwarp();
      rank[r] = before + __popc(peers & lt_mask);
    }
    __syncthreads();
    // Thread t owns digit t: tile count, warp offsets (in place), look-back.
    {
      const int d = threadIdx.x;
      uint32_t tot = 0;
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = warp_cnt[w][d];
        warp_cnt[w][d] = tot;
        tot += c;
      }
      unsigned long long* my = status + (size_t)tile * kRadix + d;
      const unsigned long long ep = (unsigned long long)(epoch & 0x3fffffffu) << 32;
      unsigned long long excl = 0;
      if (tile == 0) {
        st_release_u64(my, kFlagPrefix | ep | tot);
      } else {
        st_release_u64(my, kFlagAgg | ep | tot);
        // Batched look-back: the status words of up to kLookback predecessors
        // are loaded together (one round trip), then consumed nearest first
        // until a published prefix; a not-yet-published predecessor restarts
        // the batch from it.
        constexpr int kLookback = 16;
        int64_t j = (int64_t)tile - 1;
        const uint64_t t0 = global_ns();
        bool timed_out = false;
        while (j >= 0) {
          unsigned long long sw[kLookback];
#pragma unroll
          for (int q = 0; q < kLookback; ++q)
            sw[q] = (j - q >= 0) ? ld_acquire_u64(status + (size_t)(j - q) * kRadix + d) : 0ull;
          int q = 0;
          bool found = false;
          for (; q < kLookback && j - q >= 0; ++q) {
            const unsigned long long s = sw[q];
            const bool ready = (s & (3ull << 62)) != 0 && ((s >> 32) & 0x3fffffffull) == (epoch & 0x3fffffffu);
            if (!ready) break;
            excl += s & 0xffffffffull;
            if (s & kFlagPrefix) {
              found = true;
              break;
            }
          }
          if (found) break;
          j -= q;
          if (q == 0 && global_ns() - t0 > kWaitLimitNs) {
            timed_out = true;
            break;
          }
        }
        if (timed_out) raise_error(err, kErrSpinTimeout);
        st_release_u64(my, kFlagPrefix | ep | (excl + tot));
      }
      tile_base[d] = digit_base[d] + excl;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
      const uint32_t d = dig[r];
      if (d < 0x100u) {
        const unsigned long long pos = tile_base[d] + warp_cnt[warp][d] + rank[r];
        if (pos < (unsigned long long)n) {
          kout[pos] = key[r];
          vout[pos] = val[r];
        } else {
          raise_error(err, kErrOutputOverflow);
        }
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ top-k (K6) --
// Radix select: the k smallest keys all have a top digit <= d*, the smallest
// digit whose cumulative count reaches k.  One histogram pass over the top
// digit (its last block finds d* and the threshold), one filter pass that
// compacts the candidates (keys below the threshold), then the candidates --
// usually a few hundred -- are sorted: inside one CTA when they fit in a tile
// (a stable 8-bit LSD counting sort in shared memory), otherwise by the
// onesweep passes.  Keys are unique (packed count and id), so the first k of
// the sorted candidates are exactly the first k of the full order.
constexpr int kTopkBlock = 256;

struct TopkState {
  unsigned long long threshold;  // candidates: select digit <= threshold
  unsigned long long shift;      // bit position of the select digit
  unsigned long long n_cand;     // compacted candidates
  unsigned long long small;      // 1 when the candidates fit one CTA tile
  uint32_t done;                 // ticket for the histogram's last block
  uint32_t pad;
  unsigned long long hist[kRadix];
};

// The select digit: by default the top digit of the key; with (lo_bits,
// hi_max_dev) the key is (hi << lo_bits) | lo where every hi has the same bits
// above the highest bit of *hi_max_dev (keys packed as (cmax - count) << wa |
// id), and the digit just below that bit is the first one that orders them.
__device__ __forceinline__ int topk_shift(int top_shift, int lo_bits, const unsigned long long* hi_max_dev) {
  if (!hi_max_dev) return top_shift;
  const unsigned long long m = *hi_max_dev;
  const int L = m ? 64 - __clzll((long long)m) : 0;
  const int s = lo_bits + (L > 8 ? L - 8 : 0);
  return s < top_shift ? s : top_shift;
}

__global__ void __launch_bounds__(kTopkBlock) topk_hist_kernel(const unsigned long long* __restrict__ keys,
                                                              int64_t n_max, const unsigned long long* __restrict__ n_dev,
                                                              int top_shift_default, int lo_bits,
                                                              const unsigned long long* __restrict__ hi_max_dev, int k,
                                                              TopkState* st) {
  const int64_t n = sort_n(n_max, n_dev);
  const int top_shift = topk_shift(top_shift_default, lo_bits, hi_max_dev);
  __shared__ uint32_t h[kRadix];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  const int64_t n_w = (n + 31) & ~int64_t(31);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_w; i += stride) {
    // Warp-aggregated increments: most keys share a few top digits.
    const uint32_t d = i < n ? (uint32_t)((keys[i] >> top_shift) & 0xffu) : 0x100u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    if (d < 0x100u && lane == __ffs(peers) - 1) atomicAdd(&h[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  if (h[threadIdx.x]) atomicAdd(&st->hist[threadIdx.x], (unsigned long long)h[threadIdx.x]);
  if (!last_block(&st->done)) return;
  // Inclusive scan of the 256 bins (one per thread), then the first digit
  // whose cumulative count reaches k.
  __shared__ unsigned long long cum[kRadix];
  __shared__ int first;
  unsigned long long x = __ldcg(&st->hist[threadIdx.x]);
  cum[threadIdx.x] = x;
  if (threadIdx.x == 0) first = kRadix;
  __syncthreads();
  for (int o = 1; o < kRadix; o <<= 1) {
    const unsigned long long y = threadIdx.x >= o ? cum[threadIdx.x - o] : 0ull;
    __syncthreads();
    x += y;
    cum[threadIdx.x] = x;
    __syncthreads();
  }
  if (x >= (unsigned long long)k) atomicMin(&first, (int)threadIdx.x);
  __syncthreads();
  if (threadIdx.x == 0) {
    // keys whose select digit is <= first (all keys when the count never reaches k)
    st->threshold = (unsigned long long)(first >= kRadix ? kRadix - 1 : first);
    st->shift = (unsigned long long)top_shift;
    st->n_cand = 0;
  }
}

__global__ void __launch_bounds__(kTopkBlock) topk_filter_kernel(const unsigned long long* __restrict__ keys,
                                                                const uint32_t* __restrict__ vals, int64_t n_max,
                                                                const unsigned long long* __restrict__ n_dev,
                                                                TopkState* st, unsigned long long* __restrict__ ck,
                                                                uint32_t* __restrict__ cv) {
  const int64_t n = sort_n(n_max, n_dev);
  const unsigned long long thr = __ldcg(&st->threshold);
  const int shift = (int)__ldcg(&st->shift);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  const int64_t n_w = (n + 31) & ~int64_t(31);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_w; i += stride) {
    const unsigned long long key = i < n ? keys[i] : ~0ull;
    const bool take = i < n && ((key >> shift) & 0xffull) <= thr;
    const uint32_t ballot = __ballot_sync(0xffffffffu, take);
    if (!ballot) continue;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&st->n_cand, (unsigned long long)__popc(ballot));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (take) {
      const unsigned long long pos = base + __popc(ballot & ((1u << lane) - 1u));
      if (pos < (unsigned long long)n_max) {
        ck[pos] = key;
        cv[pos] = vals[i];
      }
    }
  }
}

// Stable LSD radix sort of <= kBlockSortMax pairs inside one CTA (8-bit digits
// over [begin_bit, end_bit)), with the same warp ranking as the onesweep pass
// (each warp owns a contiguous segment, rounds and lanes in input order).
// Sets st->small = 0 and leaves the data alone if there are more candidates
// (the onesweep passes then sort them).
constexpr int kBlockSortMax = 2048;
constexpr int kBlockSortRounds = kBlockSortMax / kSortBlock;  // keys per lane

__global__ void __launch_bounds__(kSortBlock) block_sort_kernel(unsigned long long* __restrict__ ck,
                                                                uint32_t* __restrict__ cv, TopkState* st,
                                                                int begin_bit, int end_bit) {
  extern __shared__ __align__(16) unsigned char bs_smem[];
  unsigned long long* sk = reinterpret_cast<unsigned long long*>(bs_smem);       // [2][kBlockSortMax]
  uint32_t* sv = reinterpret_cast<uint32_t*>(sk + 2 * kBlockSortMax);           // [2][kBlockSortMax]
  __shared__ uint32_t warp_cnt[kSortWarps][kRadix];
  __shared__ uint32_t dig_base[kRadix];
  const unsigned long long n = __ldcg(&st->n_cand);
  if (n > (unsigned long long)kBlockSortMax) {
    if (threadIdx.x == 0) st->small = 0;
    return;
  }
  if (threadIdx.x == 0) st->small = 1;
  for (unsigned long long i = threadIdx.x; i < n; i += blockDim.x) {
    sk[i] = ck[i];
    sv[i] = cv[i];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt_mask = (1u << lane) - 1u;
  int src = 0;
  for (int shift = begin_bit; shift < end_bit; shift += 8) {
    for (int i = threadIdx.x; i < kSortWarps * kRadix; i += blockDim.x) (&warp_cnt[0][0])[i] = 0;
    __syncthreads();
    const unsigned long long* ks = sk + src * kBlockSortMax;
    const uint32_t* vs = sv + src * kBlockSortMax;
    uint32_t rank[kBlockSortRounds], dig[kBlockSortRounds];
#pragma unroll
    for (int r = 0; r < kBlockSortRounds; ++r) {
      const unsigned long long idx = (unsigned long long)warp * (32 * kBlockSortRounds) + r * 32 + lane;
      const bool valid = idx < n;
      const uint32_t d = valid ? (uint32_t)((ks[idx] >> shift) & 0xffu) : 0x100u;
      dig[r] = d;
      const uint32_t peers = __match_any_sync(0xffffffffu, d);
      const uint32_t before = valid ? warp_cnt[warp][d] : 0u;
      __syncwarp();
      if (valid && lane == __ffs(peers) - 1) warp_cnt[warp][d] = before + __popc(peers);
      __syncwarp();
      rank[r] = before + __popc(peers & lt_mask);
    }
    __syncthreads();
    {
      const int d = threadIdx.x;  // one digit per thread
      uint32_t tot = 0;
      for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = warp_cnt[w][d];
        warp_cnt[w][d] = tot;
        tot += c;
      }
      // exclusive scan of the digit totals across the 256 threads
      dig_base[d] = tot;
      __syncthreads();
      uint32_t x = tot;
      for (int o = 1; o < kRadix; o <<= 1) {
        const uint32_t y = d >= o ? dig_base[d - o] : 0u;
        __syncthreads();
        x += y;
        dig_base[d] = x;
        __syncthreads();
      }
      dig_base[d] = x - tot;
    }
    __syncthreads();
    unsigned long long* kd = sk + (src ^ 1) * kBlockSortMax;
    uint32_t* vd = sv + (src ^ 1) * kBlockSortMax;
#pragma unroll
    for (int r = 0; r < kBlockSortRounds; ++r) {
      const uint32_t d = dig[r];
      if (d < 0x100u) {
        const unsigned long long idx = (unsigned long long)warp * (32 * kBlockSortRounds) + r * 32 + lane;
        const uint32_t pos = dig_base[d] + warp_cnt[warp][d] + rank[r];
        kd[pos] = ks[idx];
        vd[pos] = vs[idx];
      }
    }
    __syncthreads();
    src ^= 1;
  }
  for (unsigned long long i = threadIdx.x; i < n; i += blockDim.x) {
    ck[i] = sk[src * kBlockSortMax + i];
    cv[i] = sv[src * kBlockSortMax + i];
  }
}

// Key count for the onesweep fallback: 0 when the CTA sort already handled it.
__global__ void topk_big_count_kernel(const TopkState* st, unsigned long long* big) {
  if (threadIdx.x == 0) *big = __ldcg(&st->small) ? 0ull : __ldcg(&st->n_cand);
}

}  // namespace bo

using namespace bo;

namespace {
std::atomic<uint32_t> g_sort_epoch{1};
}

namespace bo {
// Sorts (keys, vals) ascending by bits [begin_bit, end_bit) of the key, stably.
// tmp_keys / tmp_vals must hold n entries.  The sorted data ends in keys/vals.
int radix_sort_pairs(bo_ctx* ctx, unsigned long long* keys, uint32_t* vals, unsigned long long* tmp_keys,
                     uint32_t* tmp_vals, int64_t n, int begin_bit, int end_bit, const unsigned long long* n_dev) {
  if (end_bit <= begin_bit || (n <= 1 && !n_dev)) return BO_OK;
  // An even number of passes leaves the result in keys/vals; pad with a pass
  // over zero bits (a stable copy of the actual keys) rather than copying the
  // whole upper-bound buffer back.
  if (((end_bit - begin_bit + 7) / 8) % 2 == 1 && end_bit + 8 <= 64) end_bit = begin_bit + 8 * ((end_bit - begin_bit + 7) / 8 + 1);
  const int n_passes = (end_bit - begin_bit + 7) / 8;
  const int64_t tiles = (n + kSortTile - 1) / kSortTile;
  if (tiles > 0x7fffffff) return set_error(ctx, BO_ERR_INVALID, "radix_sort: too many keys");
  void* p = nullptr;
  const size_t hist_bytes = sizeof(unsigned long long) * kMaxPasses * kRadix;
  const size_t ctr_bytes = 256;
  const size_t status_bytes = sizeof(unsigned long long) * (size_t)tiles * kRadix;
  int rc = region(ctx, "sort_ws", hist_bytes + ctr_bytes + status_bytes, &p);
  if (rc) return rc;
  unsigned long long* hist = static_cast<unsigned long long*>(p);
  uint32_t* ctr = reinterpret_cast<uint32_t*>(static_cast<char*>(p) + hist_bytes);
  unsigned long long* status = reinterpret_cast<unsigned long long*>(static_cast<char*>(p) + hist_bytes + ctr_bytes);
  BO_CUDA(ctx, cudaMemsetAsync(p, 0, hist_bytes + ctr_bytes, ctx->stream));
  const int hg = (int)std::min<int64_t>((n + kSortBlock - 1) / kSortBlock, (int64_t)ctx->num_sms);
  radix_hist_kernel<<<std::max(hg, 1), kSortBlock, 0, ctx->stream>>>(keys, n, n_dev, begin_bit, n_passes, hist,
                                                                      ctr + kMaxPasses);
  if ((rc = after_launch(ctx, "radix_hist_kernel"))) return rc;
  const int64_t resident = (int64_t)ctx->num_sms *
                           occupancy_blocks(reinterpret_cast<const void*>(&radix_pass_kernel), kSortBlock, 0);
  const int pass_grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, resident));
  unsigned long long *src_k = keys, *dst_k = tmp_keys;
  uint32_t *src_v = vals, *dst_v = tmp_vals;
  for (int pass = 0; pass < n_passes; ++pass) {
    const uint32_t epoch = g_sort_epoch.fetch_add(1);
    radix_pass_kernel<<<pass_grid, kSortBlock, 0, ctx->stream>>>(src_k, src_v, dst_k, dst_v, n, n_dev,
                                                                    begin_bit + 8 * pass, hist + pass * kRadix, status,
                                                                    ctr + pass, epoch, ctx->d_err);
    if ((rc = after_launch(ctx, "radix_pass_kernel"))) return rc;
    std::swap(src_k, dst_k);
    std::swap(src_v, dst_v);
  }
  if (src_k != keys) {
    BO_CUDA(ctx, cudaMemcpyAsync(keys, src_k, sizeof(unsigned long long) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    BO_CUDA(ctx, cudaMemcpyAsync(vals, src_v, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  return BO_OK;
}
}  // namespace bo

namespace bo {
// The k smallest keys in ascending order, written to the front of
// (cand_keys, cand_vals) (capacity n_max each); the count of keys comes from
// n_dev.  Asynchronous; no host round trip.
int radix_topk_pairs(bo_ctx* ctx, const unsigned long long* keys, const uint32_t* vals, int64_t n_max,
                     const unsigned long long* n_dev, int key_bits, int k, unsigned long long* cand_keys,
                     uint32_t* cand_vals, unsigned long long* tmp_keys, uint32_t* tmp_vals, int lo_bits,
                     const unsigned long long* hi_max_dev) {
  void* p = nullptr;
  int rc = region(ctx, "topk_state", sizeof(TopkState), &p);
  if (rc) return rc;
  TopkState* st = static_cast<TopkState*>(p);
  BO_CUDA(ctx, cudaMemsetAsync(st, 0, sizeof(TopkState), ctx->stream));
  const int bits = std::max(8, ((key_bits + 7) / 8) * 8);
  const int top_shift = bits - 8;
  const int g = (int)std::max<int64_t>(1, std::min<int64_t>((n_max + kTopkBlock - 1) / kTopkBlock, ctx->num_sms));
  topk_hist_kernel<<<g, kTopkBlock, 0, ctx->stream>>>(keys, n_max, n_dev, top_shift, lo_bits, hi_max_dev,
                                                       std::max(k, 1), st);
  if ((rc = after_launch(ctx, "topk_hist_kernel"))) return rc;
  topk_filter_kernel<<<g, kTopkBlock, 0, ctx->stream>>>(keys, vals, n_max, n_dev, st, cand_keys, cand_vals);
  if ((rc = after_launch(ctx, "topk_filter_kernel"))) return rc;
  const size_t bs_smem = (sizeof(unsigned long long) + sizeof(uint32_t)) * 2 * kBlockSortMax;
  static bool bs_ready = false;
  if (!bs_ready) {
    BO_CUDA(ctx, cudaFuncSetAttribute(reinterpret_cast<const void*>(&block_sort_kernel),
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bs_smem));
    bs_ready = true;
  }
  block_sort_kernel<<<1, kSortBlock, bs_smem, ctx->stream>>>(cand_keys, cand_vals, st, 0, bits);
  if ((rc = after_launch(ctx, "block_sort_kernel"))) return rc;
  // Large candidate sets (heavy ties in the top digit): the onesweep passes.
  // With a small set they see a zero count and retire immediately.
  void* q = nullptr;
  if ((rc = region(ctx, "topk_bigcount", 64, &q))) return rc;
  unsigned long long* big = static_cast<unsigned long long*>(q);
  topk_big_count_kernel<<<1, 32, 0, ctx->stream>>>(st, big);
  if ((rc = after_launch(ctx, "topk_big_count_kernel"))) return rc;
  return radix_sort_pairs(ctx, cand_keys, cand_vals, tmp_keys, tmp_vals, n_max, 0, bits, big);
}
}  // namespace bo

extern "C" {

int bo_radix_sort_pairs_device(bo_ctx* ctx, uint64_t* keys, uint32_t* vals, int64_t n, int32_t begin_bit,
                               int32_t end_bit) {
  BO_CHECK_CTX(ctx);
  if (n < 0 || (n > 0 && (!keys || !vals)) || begin_bit < 0 || end_bit > 64 || begin_bit > end_bit)
    return set_error(ctx, BO_ERR_INVALID, "radix_sort: bad argument");
  if (n <= 1) return BO_OK;
  void* tmp = nullptr;
  const size_t kb = (sizeof(unsigned long long) * (size_t)n + 255) & ~size_t(255);
  int rc = region(ctx, "sort_tmp", kb + sizeof(uint32_t) * (size_t)n, &tmp);
  if (rc) return rc;
  return radix_sort_pairs(ctx, reinterpret_cast<unsigned long long*>(keys), vals,
                          static_cast<unsigned long long*>(tmp),
                          reinterpret_cast<uint32_t*>(static_cast<char*>(tmp) + kb), n, begin_bit, end_bit, nullptr);
}

int bo_radix_sort_pairs_host(bo_ctx* ctx, uint64_t* keys, uint32_t* vals, int64_t n, int32_t begin_bit,
                             int32_t end_bit) {
  BO_CHECK_CTX(ctx);
  if (n < 0 || (n > 0 && (!keys || !vals))) return set_error(ctx, BO_ERR_INVALID, "radix_sort: bad argument");
  if (n == 0) return BO_OK;
  void* buf = nullptr;
  const size_t kb = (sizeof(unsigned long long) * (size_t)n + 255) & ~size_t(255);
  int rc = region(ctx, "sort_in", kb + sizeof(uint32_t) * (size_t)n, &buf);
  if (rc) return rc;
  uint64_t* dk = static_cast<uint64_t*>(buf);
  uint32_t* dv = reinterpret_cast<uint32_t*>(static_cast<char*>(buf) + kb);
  BO_CUDA(ctx, cudaMemcpyAsync(dk, keys, sizeof(uint64_t) * n, cudaMemcpyHostToDevice, ctx->stream));
  BO_CUDA(ctx, cudaMemcpyAsync(dv, vals, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = bo_radix_sort_pairs_device(ctx, dk, dv, n, begin_bit, end_bit))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(keys, dk, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaMemcpyAsync(vals, dv, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;
  return device_error_status(ctx, bits, "radix_sort");
}

}  // extern "C"
