// LSD onesweep radix sort of (uint64 key, uint32 value) pairs with decoupled
// look-back (K5), a one-launch cluster sort for up to 128K pairs, and top-k by
// radix select (K6).
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
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "context.cuh"

namespace cg = cooperative_groups;

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
// The k smallest of n unique keys (packed count and id) in one cooperative
// launch: an exact radix select, 8 bits per round from the key's highest
// varying digit down.  Each round every block histograms the digit of the keys
// that still match the selected prefix (shared-memory counters, one global
// atomic per bin per block), a grid barrier, and every block finds the same
// digit where the cumulative count reaches the number of keys still needed.
// When that digit's bin holds exactly the keys still needed, or after the last
// digit, the selected keys are those at or below the prefix: they are
// compacted (at most k <= 64), and block 0 orders them by rank.  The grid
// barriers spin on a generation word bounded by the global timer (a timeout
// sets an error bit); cooperative launch keeps every block resident.
constexpr int kSelBlock = 256;
constexpr int kSelMaxK = 64;
constexpr int kSelMaxRounds = 8;

struct SelectState {
  unsigned long long hist[kSelMaxRounds][kRadix];
  unsigned long long n_sel;
  uint32_t bar_count;
  uint32_t bar_gen;
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


__device__ __forceinline__ void grid_barrier(SelectState* st, uint32_t& bad) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t g = ld_acquire_u32(&st->bar_gen);
    __threadfence();
    if (atomicAdd(&st->bar_count, 1u) == gridDim.x - 1) {
      st->bar_count = 0;
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    } else {
      const uint64_t t0 = global_ns();
      while (ld_acquire_u32(&st->bar_gen) == g) {
        if (global_ns() - t0 > kWaitLimitNs) {
          bad |= kErrSpinTimeout;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kSelBlock) topk_select_kernel(const unsigned long long* __restrict__ keys,
                                                               const uint32_t* __restrict__ vals, int64_t n_max,
                                                               const unsigned long long* __restrict__ n_dev,
                                                               int top_shift_default, int lo_bits,
                                                               const unsigned long long* __restrict__ hi_max_dev,
                                                               int k, SelectState* st, unsigned long long* __restrict__ ck,
                                                               uint32_t* __restrict__ cv, uint32_t* err) {
  const int64_t n = sort_n(n_max, n_dev);
  const int64_t kk = k < kSelMaxK ? (int64_t)k : (int64_t)kSelMaxK;
  const unsigned long long want = (unsigned long long)(n < kk ? n : kk);
  if (want == 0) return;  // the same in every block
  // Keys lie below 2^(s0 + 8): every bit above the first digit is zero.
  const int s0 = topk_shift(top_shift_default, lo_bits, hi_max_dev);
  __shared__ uint32_t h[kRadix];
  __shared__ unsigned long long cum[kRadix];
  __shared__ int first;
  const int t = threadIdx.x, lane = t & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t n_w = (n + 31) & ~int64_t(31);
  uint32_t bad = 0;
  unsigned long long prefix = 0, pmask = 0, need = want;
  int round = 0;
  for (int sh = s0; sh > -8 && round < kSelMaxRounds; sh -= 8, ++round) {
    const int shift = sh < 0 ? 0 : sh;
    const unsigned long long dmask = (1ull << (sh < 0 ? sh + 8 : 8)) - 1ull;
    h[t] = 0;
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + t; i < n_w; i += stride) {
      const unsigned long long key = i < n ? keys[i] : 0ull;
      const uint32_t d = (i < n && (key & pmask) == prefix) ? (uint32_t)((key >> shift) & dmask) : 0x100u;
      const uint32_t peers = __match_any_sync(0xffffffffu, d);
      if (d < 0x100u && lane == __ffs(peers) - 1) atomicAdd(&h[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    if (h[t]) atomicAdd(&st->hist[round][t], (unsigned long long)h[t]);
    grid_barrier(st, bad);
    // Inclusive scan of the round's bins (one per thread); the first digit
    // whose cumulative count reaches `need`.
    const unsigned long long own = __ldcg(&st->hist[round][t]);
    unsigned long long x = own;
    cum[t] = x;
    if (t == 0) first = kRadix;
    __syncthreads();
    for (int o = 1; o < kRadix; o <<= 1) {
      const unsigned long long y = t >= o ? cum[t - o] : 0ull;
      __syncthreads();
      x += y;
      cum[t] = x;
      __syncthreads();
    }
    if (x >= need) atomicMin(&first, t);
    __syncthreads();
    const int dg = first < kRadix ? first : kRadix - 1;  // (always found: the matching keys number >= need)
    const unsigned long long below = dg > 0 ? cum[dg - 1] : 0ull;
    const unsigned long long at = cum[dg] - below;
    __syncthreads();
    need -= below;
    prefix |= (unsigned long long)dg << shift;
    pmask |= dmask << shift;
    if (at == need) break;  // every key of this digit is taken: the prefix decides
  }
  // Selected: the keys whose bits under pmask are at or below the prefix.
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + t; i < n_w; i += stride) {
    const unsigned long long key = i < n ? keys[i] : ~0ull;
    const bool take = i < n && (key & pmask) <= prefix;
    const uint32_t ballot = __ballot_sync(0xffffffffu, take);
    if (!ballot) continue;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&st->n_sel, (unsigned long long)__popc(ballot));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (take) {
      const unsigned long long pos = base + __popc(ballot & ((1u << lane) - 1u));
      if (pos < (unsigned long long)kSelMaxK) {
        ck[pos] = key;
        cv[pos] = vals[i];
      } else {
        bad |= kErrOutputOverflow;
      }
    }
  }
  grid_barrier(st, bad);
  if (blockIdx.x == 0) {
    __shared__ unsigned long long sk[kSelMaxK];
    __shared__ uint32_t sv[kSelMaxK];
    const unsigned long long ns = __ldcg(&st->n_sel);
    const int m = (int)(ns < (unsigned long long)kSelMaxK ? ns : (unsigned long long)kSelMaxK);
    if (ns != want) bad |= kErrOutputOverflow;
    if (t < m) {
      sk[t] = ck[t];
      sv[t] = cv[t];
    }
    __syncthreads();
    if (t < m) {  // unique keys: the rank is the count of smaller keys
      int r = 0;
      for (int j = 0; j < m; ++j) r += sk[j] < sk[t];
      ck[r] = sk[t];
      cv[r] = sv[t];
    }
  }
  if (bad) raise_error(err, bad);
}

// Lanes of the warp holding the same digit (0..0x100, 0x100 = no row), from
// 9 ballots (measured faster than __match_any_sync in the sort below).
__device__ __forceinline__ uint32_t digit_peers(uint32_t d) {
  uint32_t m = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < 9; ++b) {
    const uint32_t bit = (d >> b) & 1u;
    const uint32_t bal = __ballot_sync(0xffffffffu, bit);
    m &= bit ? bal : ~bal;
  }
  return m;
}

// Stable LSD radix sort of up to kClusterSortMax pairs by one thread-block
// cluster, the pairs held in the CTAs' shared memory for the whole sort: CTA
// r holds global positions [r*S, r*S + S).  Per 8-bit digit every warp ranks
// its contiguous 512-pair segment (rounds and lanes in input order, as the
// onesweep pass), each CTA publishes its 256 digit totals, every CTA reads the
// cluster's totals through distributed shared memory to place its digits, and
// each pair is stored straight into the shared memory of the CTA that owns
// its destination (st.shared::cluster); one cluster barrier per digit.  A
// digit that every key shares is skipped.  No global memory between the load
// and the final store, one launch for the whole sort.
constexpr int kCsBlock = 512;
constexpr int kCsWarps = kCsBlock / 32;
constexpr int kCsCap = 8192;                    // pairs per CTA
constexpr int kCsRounds = kCsCap / kCsBlock;    // rounds of 32 per warp
constexpr int kCsPortable = 8;                  // portable cluster size
constexpr int kCsMaxCluster = 16;               // non-portable, where the device schedules it
constexpr int64_t kCsTargetPerCta = 1024;       // spread: about this many pairs per CTA
constexpr int64_t kClusterSortMax = (int64_t)kCsCap * kCsMaxCluster;
constexpr size_t kCsDynSmem = (size_t)2 * kCsCap * (sizeof(unsigned long long) + sizeof(uint32_t));

// n_dev (optional): the count is min(*n_dev, n), read on the device; a count
// beyond the cluster's capacity sets *overflow and sorts nothing (every CTA
// reads the same count, so all return before the first cluster barrier).
__global__ void __launch_bounds__(kCsBlock, 1) cluster_sort_kernel(unsigned long long* __restrict__ keys,
                                                                  uint32_t* __restrict__ vals, int64_t n,
                                                                  int begin_bit, int end_bit,
                                                                  const unsigned long long* __restrict__ n_dev,
                                                                  uint32_t* __restrict__ overflow) {
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t cs = cl.num_blocks();
  const uint32_t me = cl.block_rank();
  if (n_dev) {
    const unsigned long long nd = *n_dev;
    if (nd < (unsigned long long)n) n = (int64_t)nd;
    if (n > (int64_t)kCsCap * cs) {
      if (me == 0 && threadIdx.x == 0) atomicOr(overflow, 1u);
      return;
    }
  }
  extern __shared__ __align__(16) unsigned char cs_smem[];
  // [2][S] keys then [2][S] values: the launch sizes the dynamic shared
  // memory to the pairs per CTA (S <= kCsCap), not to the capacity.
  unsigned long long* sk = reinterpret_cast<unsigned long long*>(cs_smem);
  __shared__ uint32_t warp_cnt[kCsWarps][kRadix];
  __shared__ uint32_t tot[kRadix];   // this CTA's digit totals, read by the whole cluster
  __shared__ uint32_t base[kRadix];  // where this CTA's pairs of each digit start
  __shared__ uint32_t wsum[kRadix / 32];
  __shared__ int skip;
  const uint32_t S = (uint32_t)((n + cs - 1) / cs);  // <= kCsCap (checked by the host)
  uint32_t* sv = reinterpret_cast<uint32_t*>(sk + 2 * S);
  const int64_t lo = (int64_t)me * S;
  const int64_t left = n - lo;
  const uint32_t m = left <= 0 ? 0u : (left < (int64_t)S ? (uint32_t)left : S);
  for (uint32_t i = threadIdx.x; i < m; i += kCsBlock) {
    sk[i] = keys[lo + i];
    sv[i] = vals[lo + i];
  }
  cl.sync();  // every CTA runs (and has loaded) before any pair moves between them
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt_mask = (1u << lane) - 1u;
  // Warp segments of `seg` pairs (a multiple of 32, the same in every CTA):
  // only as many rounds as the CTA's pairs need.
  const uint32_t seg = ((S + kCsWarps * 32 - 1) / (kCsWarps * 32)) * 32;
  const int rounds = (int)(seg / 32);
  int src = 0;
  for (int shift = begin_bit; shift < end_bit; shift += 8) {
    const uint32_t dmask = (1u << min(8, end_bit - shift)) - 1u;
    for (int i = threadIdx.x; i < kCsWarps * kRadix; i += kCsBlock) (&warp_cnt[0][0])[i] = 0;
    if (threadIdx.x == 0) skip = 0;
    __syncthreads();
    const unsigned long long* ks = sk + src * S;
    const uint32_t* vs = sv + src * S;
    uint32_t rank[kCsRounds], dig[kCsRounds];
#pragma unroll
    for (int r = 0; r < kCsRounds; ++r) {
      dig[r] = 0x100u;
      rank[r] = 0;
      if (r >= rounds) continue;  // the same for every lane of the warp
      const uint32_t idx = (uint32_t)warp * seg + r * 32 + lane;
      const bool valid = idx < m;
      const uint32_t d = valid ? (uint32_t)((ks[idx] >> shift) & dmask) : 0x100u;
      dig[r] = d;
      const uint32_t peers = digit_peers(d);
      const uint32_t before = valid ? warp_cnt[warp][d] : 0u;
      __syncwarp();
      if (valid && lane == __ffs(peers) - 1) warp_cnt[warp][d] = before + __popc(peers);
      __syncwarp();
      rank[r] = before + __popc(peers & lt_mask);
    }
    __syncthreads();
    if (threadIdx.x < kRadix) {  // one digit per thread: warps' exclusive prefix, CTA total
      const int d = threadIdx.x;
      uint32_t t = 0;
      for (int w = 0; w < kCsWarps; ++w) {
        const uint32_t c = warp_cnt[w][d];
        warp_cnt[w][d] = t;
        t += c;
      }
      tot[d] = t;
    }
    cl.sync();  // every CTA's totals are published
    uint32_t all = 0, below = 0, incl = 0;
    if (threadIdx.x < kRadix) {
      const int d = threadIdx.x;
      for (uint32_t q = 0; q < cs; ++q) {
        const uint32_t v = cl.map_shared_rank(tot, q)[d];
        all += v;
        if (q < me) below += v;
      }
      incl = all;  // inclusive scan over the digits: within the warp, then across the 8 warps
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) wsum[warp] = incl;
      if (all == (uint32_t)n) skip = 1;  // every key has this digit: the pass would not move anything
    }
    __syncthreads();
    if (threadIdx.x < kRadix) {
      uint32_t pre = 0;
      for (int w = 0; w < warp; ++w) pre += wsum[w];
      base[threadIdx.x] = pre + incl - all + below;
    }
    __syncthreads();
    if (!skip) {
      unsigned long long* kd = sk + (src ^ 1) * S;
      uint32_t* vd = sv + (src ^ 1) * S;
#pragma unroll
      for (int r = 0; r < kCsRounds; ++r) {
        const uint32_t d = dig[r];
        if (d < 0x100u) {
          const uint32_t idx = (uint32_t)warp * seg + r * 32 + lane;
          const uint32_t pos = base[d] + warp_cnt[warp][d] + rank[r];
          const uint32_t q = pos / S, slot = pos - q * S;
          cl.map_shared_rank(kd, q)[slot] = ks[idx];
          cl.map_shared_rank(vd, q)[slot] = vs[idx];
        }
      }
    }
    cl.sync();  // all pairs placed and all totals read before the next digit
    if (!skip) src ^= 1;
  }
  for (uint32_t i = threadIdx.x; i < m; i += kCsBlock) {
    keys[lo + i] = sk[src * S + i];
    vals[lo + i] = sv[src * S + i];
  }
}

}  // namespace bo

using namespace bo;

namespace {
std::atomic<uint32_t> g_sort_epoch{1};
}

namespace bo {
// Sorts (keys, vals) ascending by bits [begin_bit, end_bit) of the key, stably.
// tmp_keys / tmp_vals must hold n entries.  The sorted data ends in keys/vals.
// One cluster of the smallest power-of-two size whose shared memory holds the
// pairs (n <= kClusterSortMax).
// The largest cluster the device schedules for the sort: 16 CTAs where a
// non-portable cluster of that size fits (B200), else 8.  Checked once.
int cluster_sort_max(bo_ctx* ctx) {
  static int cached = 0;
  if (cached) return cached;
  if (cudaFuncSetAttribute(cluster_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCsDynSmem) !=
      cudaSuccess) {
    cudaGetLastError();
    return kCsPortable;
  }
  int best = kCsPortable;
  if (cudaFuncSetAttribute(cluster_sort_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kCsMaxCluster);
    cfg.blockDim = dim3(kCsBlock);
    cfg.dynamicSmemBytes = kCsDynSmem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kCsMaxCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, reinterpret_cast<const void*>(&cluster_sort_kernel), &cfg) ==
            cudaSuccess &&
        clusters >= 1)
      best = kCsMaxCluster;
  }
  cudaGetLastError();
  (void)ctx;
  cached = best;
  return cached;
}

int cluster_sort_pairs(bo_ctx* ctx, unsigned long long* keys, uint32_t* vals, int64_t n, int begin_bit,
                       int end_bit) {
  if (n <= 1 || end_bit <= begin_bit) return BO_OK;
  const int max_cs = cluster_sort_max(ctx);
  if (n > (int64_t)kCsCap * max_cs) return set_error(ctx, BO_ERR_INVALID, "cluster_sort: %lld pairs", (long long)n);
  // Enough CTAs to hold the pairs, and more (up to the largest cluster) so
  // that each CTA ranks about kCsTargetPerCta of them: one CTA's passes are
  // instruction-bound, so the sort takes time in proportion to its share.
  unsigned cs = 1;
  while ((int64_t)cs * kCsCap < n) cs <<= 1;
  while ((int)cs < max_cs && (int64_t)cs * kCsTargetPerCta < n) cs <<= 1;
  static bool ready = false;
  if (!ready) {
    BO_CUDA(ctx, cudaFuncSetAttribute(cluster_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kCsDynSmem));
    ready = true;
  }
  const int64_t per_cta = (n + cs - 1) / cs;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs);
  cfg.blockDim = dim3(kCsBlock);
  cfg.dynamicSmemBytes = (size_t)2 * per_cta * (sizeof(unsigned long long) + sizeof(uint32_t));
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BO_CUDA(ctx, cudaLaunchKernelEx(&cfg, cluster_sort_kernel, keys, vals, n, begin_bit, end_bit,
                                  static_cast<const unsigned long long*>(nullptr), static_cast<uint32_t*>(nullptr)));
  return after_launch(ctx, "cluster_sort_kernel");
}

int cluster_sort_pairs_counted(bo_ctx* ctx, unsigned long long* keys, uint32_t* vals, const unsigned long long* n_dev,
                               int64_t n_max, int begin_bit, int end_bit, uint32_t* overflow) {
  if (n_max <= 1 || end_bit <= begin_bit) return BO_OK;
  const int max_cs = cluster_sort_max(ctx);
  static bool ready = false;
  if (!ready) {
    BO_CUDA(ctx, cudaFuncSetAttribute(cluster_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kCsDynSmem));
    ready = true;
  }
  // The count is unknown here: the largest cluster, each CTA with room for
  // its capacity, so any count up to kCsCap * max_cs fits.
  unsigned cs = 1;
  while ((int)cs < max_cs && (int64_t)cs * kCsTargetPerCta < n_max) cs <<= 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs);
  cfg.blockDim = dim3(kCsBlock);
  cfg.dynamicSmemBytes = kCsDynSmem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BO_CUDA(ctx, cudaLaunchKernelEx(&cfg, cluster_sort_kernel, keys, vals, n_max, begin_bit, end_bit, n_dev, overflow));
  return after_launch(ctx, "cluster_sort_kernel");
}

void* mapped_device_ptr(const void* host) {
  if (!host) return nullptr;
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, host) != cudaSuccess) {
    cudaGetLastError();  // not a pointer CUDA knows: pageable memory
    return nullptr;
  }
  if (attr.type != cudaMemoryTypeHost || !attr.devicePointer || !aligned16(attr.devicePointer)) return nullptr;
  return attr.devicePointer;
}

int read_counted(bo_ctx* ctx, const char* op, const unsigned long long* n_out, int64_t n_max, int64_t* n,
                 bool* overflow) {
  BO_CUDA(ctx, cudaMemcpyAsync(ctx->h_word, n_out, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                               ctx->stream));
  uint32_t bits = 0;
  int rc = consume_device_errors(ctx, &bits);  // synchronises the stream
  if (rc) return rc;
  if ((rc = device_error_status(ctx, bits, op))) return rc;
  *n = (int64_t)std::min<unsigned long long>(ctx->h_word[0], (unsigned long long)std::max<int64_t>(n_max, 0));
  *overflow = (uint32_t)ctx->h_word[1] != 0u;
  return BO_OK;
}

int read_device_count(bo_ctx* ctx, const unsigned long long* n_dev, int64_t n_max, int64_t* n) {
  BO_CUDA(ctx, cudaMemcpyAsync(ctx->h_word, n_dev, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *n = (int64_t)std::min<unsigned long long>(*ctx->h_word, (unsigned long long)std::max<int64_t>(n_max, 0));
  return BO_OK;
}

int radix_sort_pairs(bo_ctx* ctx, unsigned long long* keys, uint32_t* vals, unsigned long long* tmp_keys,
                     uint32_t* tmp_vals, int64_t n, int begin_bit, int end_bit, const unsigned long long* n_dev) {
  if (end_bit <= begin_bit || (n <= 1 && !n_dev)) return BO_OK;
  if (!n_dev && n <= (int64_t)kCsCap * cluster_sort_max(ctx))
    return cluster_sort_pairs(ctx, keys, vals, n, begin_bit, end_bit);
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
// The k smallest keys (k <= 64; the keys must be unique) in ascending order,
// written to the front of (cand_keys, cand_vals); the count of keys comes
// from n_dev.  One memset and one cooperative launch; no host round trip.
int radix_topk_pairs(bo_ctx* ctx, const unsigned long long* keys, const uint32_t* vals, int64_t n_max,
                     const unsigned long long* n_dev, int key_bits, int k, unsigned long long* cand_keys,
                     uint32_t* cand_vals, unsigned long long* tmp_keys, uint32_t* tmp_vals, int lo_bits,
                     const unsigned long long* hi_max_dev) {
  (void)tmp_keys;
  (void)tmp_vals;
  if (k < 0 || k > kSelMaxK) return set_error(ctx, BO_ERR_INVALID, "top-k: k = %d outside [0, %d]", k, kSelMaxK);
  void* p = nullptr;
  int rc = region(ctx, "topk_select", sizeof(SelectState), &p);
  if (rc) return rc;
  SelectState* st = static_cast<SelectState*>(p);
  BO_CUDA(ctx, cudaMemsetAsync(st, 0, sizeof(SelectState), ctx->stream));
  const int bits = std::max(8, ((key_bits + 7) / 8) * 8);
  const int top_shift = std::min(bits, 64) - 8;
  const void* kf = reinterpret_cast<const void*>(&topk_select_kernel);
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(kf, kSelBlock, 0);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(resident, (n_max + 4 * kSelBlock - 1) / (4 * kSelBlock)));
  // A cooperative launch (every block resident: the grid barriers rely on it),
  // through cudaLaunchKernelEx so that stream capture records it as a graph node.
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kSelBlock);
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BO_CUDA(ctx, cudaLaunchKernelEx(&cfg, topk_select_kernel, keys, vals, n_max, n_dev, top_shift, lo_bits, hi_max_dev, k,
                                  st, cand_keys, cand_vals, ctx->d_err));
  return after_launch(ctx, "topk_select_kernel");
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
