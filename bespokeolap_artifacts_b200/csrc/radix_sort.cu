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
//    radix_scan_kernel turns them into exclusive digit bases;
//  * radix_pass_kernel -- tiles of 4096 keys, tile ids taken from an atomic
//    counter so every predecessor tile has started.  A warp ranks its 512 keys
//    stably in 16 rounds of 32 (match_any on the digit, per-warp digit counters
//    in shared memory), the block sums its warps into tile counts, publishes
//    them, and each of the 256 threads does the decoupled look-back for one
//    digit over predecessor tiles' 64-bit status words
//    (flag:2 | epoch:30 | count:32).  The epoch (unique per pass launch) makes
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

__global__ void __launch_bounds__(kSortBlock) radix_hist_kernel(const unsigned long long* __restrict__ keys, int64_t n_max,
                                                                const unsigned long long* __restrict__ n_dev,
                                                                int begin_bit, int n_passes,
                                                                unsigned long long* __restrict__ hist) {
  const int64_t n = sort_n(n_max, n_dev);
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
}

// One block: exclusive scan of each pass's 256 bins (hist -> bases, in place).
__global__ void __launch_bounds__(kRadix) radix_scan_kernel(unsigned long long* hist, int n_passes) {
  __shared__ unsigned long long s[kRadix];
  for (int p = 0; p < n_passes; ++p) {
    const unsigned long long v = hist[p * kRadix + threadIdx.x];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kRadix; o <<= 1) {
      const unsigned long long add = threadIdx.x >= o ? s[threadIdx.x - o] : 0ull;
      __syncthreads();
      s[threadIdx.x] += add;
      __syncthreads();
    }
    hist[p * kRadix + threadIdx.x] = s[threadIdx.x] - v;
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
  __shared__ uint32_t warp_cnt[kSortWarps][kRadix];
  __shared__ unsigned long long tile_base[kRadix];
  __shared__ uint32_t tile_s;
  for (int i = threadIdx.x; i < kSortWarps * kRadix; i += blockDim.x) (&warp_cnt[0][0])[i] = 0;
  if (threadIdx.x == 0) tile_s = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = tile_s;
  if ((int64_t)tile * kSortTile >= n && tile != 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t seg = (int64_t)tile * kSortTile + (int64_t)warp * (32 * kSortRounds);
  const uint32_t lt_mask = (1u << lane) - 1u;

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
      int64_t j = (int64_t)tile - 1;
      const uint64_t t0 = global_ns();
      bool timed_out = false;
      while (j >= 0) {
        const unsigned long long s = ld_acquire_u64(status + (size_t)j * kRadix + d);
        const bool ready = (s & (3ull << 62)) != 0 && ((s >> 32) & 0x3fffffffull) == (epoch & 0x3fffffffu);
        if (!ready) {
          if (global_ns() - t0 > kWaitLimitNs) {
            timed_out = true;
            break;
          }
          continue;
        }
        excl += s & 0xffffffffull;
        if (s & kFlagPrefix) break;
        --j;
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
  const int hg = (int)std::min<int64_t>((n + kSortBlock - 1) / kSortBlock, (int64_t)ctx->num_sms * 4);
  radix_hist_kernel<<<std::max(hg, 1), kSortBlock, 0, ctx->stream>>>(keys, n, n_dev, begin_bit, n_passes, hist);
  if ((rc = after_launch(ctx, "radix_hist_kernel"))) return rc;
  radix_scan_kernel<<<1, kRadix, 0, ctx->stream>>>(hist, n_passes);
  if ((rc = after_launch(ctx, "radix_scan_kernel"))) return rc;
  unsigned long long *src_k = keys, *dst_k = tmp_keys;
  uint32_t *src_v = vals, *dst_v = tmp_vals;
  for (int pass = 0; pass < n_passes; ++pass) {
    const uint32_t epoch = g_sort_epoch.fetch_add(1);
    radix_pass_kernel<<<(int)tiles, kSortBlock, 0, ctx->stream>>>(src_k, src_v, dst_k, dst_v, n, n_dev,
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
