// TPC-H Q13 over the storage-plan layout: run_q13 of
// bespoke_tpch/query_q13.cpp:166-270.
//
// The reference scans every order's comment (alpha / bigram masks first, then
// memchr + memcmp for word1 and word2, :44-83, :192-223), counts the orders
// that do not match per custkey, histograms the customers' counts and sorts
// the (c_count, custdist) pairs.  Here:
//   orders    one warp per 32 consecutive orders: their comments are one
//             contiguous byte range, staged into the warp's shared-memory
//             slice with 16-byte coalesced loads (ranges larger than the
//             slice are read in place), then each lane runs the reference's
//             two-step search on its own comment; non-matching orders add 1
//             to their customer's count (the counts stay in L2) and the warp
//             keeps the largest count it produced;
//   customers a per-block shared histogram of counts below 1024, larger
//             counts straight to the global histogram;
//   emit/sort the non-zero bins [0, max count] (cleared as they are read, so
//             the histogram needs no per-call memset) as one 64-bit key
//             (custdist desc, c_count desc) through the onesweep radix sort.
// The masks are a CPU shortcut: they only skip comments that cannot match,
// so the result does not depend on them.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "context.cuh"
#include "q13_search.cuh"

namespace bo {
namespace {

constexpr int kQ13Block = 256;
constexpr int kQ13Warps = kQ13Block / 32;
constexpr uint32_t kQ13SliceBytes = 4096;  // per warp: 32 comments of up to 128 bytes on average
constexpr int kQ13StageBatch = 2;          // 16-byte loads per lane in flight while staging
constexpr int kQ13SmallBins = 1024;

// First position p >= from with s[p, p + l) == w, else n; an empty word
// matches at `from` (find_substring, query_q13.cpp:44-66).
__device__ __forceinline__ uint32_t q13_find(const uint8_t* s, uint32_t from, uint32_t n, const uint8_t* w,
                                             uint32_t l) {
  if (l == 0) return from;
  if (n < l) return n;
  const uint8_t c0 = __ldg(w);
  for (uint32_t p = from; p + l <= n; ++p) {
    if (s[p] != c0) continue;
    uint32_t k = 1;
    while (k < l && s[p + k] == __ldg(w + k)) ++k;
    if (k == l) return p;
  }
  return n;
}

// matches_pattern (query_q13.cpp:68-83).
__device__ __forceinline__ bool q13_match(const uint8_t* s, uint32_t n, const uint8_t* w1, uint32_t l1,
                                          const uint8_t* w2, uint32_t l2) {
  const uint32_t p1 = q13_find(s, 0, n, w1, l1);
  if (p1 == n) return false;
  return q13_find(s, p1 + l1, n, w2, l2) != n;
}

__global__ void __launch_bounds__(kQ13Block) q13_orders_kernel(const uint8_t* __restrict__ data,
                                                               const uint32_t* __restrict__ offsets,
                                                               const int32_t* __restrict__ o_custkey, int64_t n,
                                                               const uint8_t* __restrict__ words, uint32_t l1,
                                                               uint32_t l2, uint32_t* __restrict__ counts,
                                                               int64_t n_counts, uint32_t* max_count, uint32_t* err) {
  __shared__ __align__(16) uint8_t slices[kQ13Warps][kQ13SliceBytes];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint8_t* slice = slices[warp];
  const uint32_t total = offsets[n];
  const uint8_t* w1 = words;
  const uint8_t* w2 = words + l1;
  uint32_t local_max = 0;
  const int64_t warps = (int64_t)gridDim.x * kQ13Warps;
  for (int64_t g = (int64_t)blockIdx.x * kQ13Warps + warp; g * 32 < n; g += warps) {
    const int64_t first = g * 32;
    const int64_t last = min(first + 32, n);
    const int64_t i = first + lane;
    // Independent loads first: this lane's bounds and custkey, the group's byte range.
    uint32_t s0 = 0, s1 = 0;
    int32_t c = 0;
    if (i < last) {
      s0 = offsets[i];
      s1 = offsets[i + 1];
      c = o_custkey[i];
    }
    const uint32_t b0 = __shfl_sync(0xffffffffu, s0, 0);
    const uint32_t b1 = __shfl_sync(0xffffffffu, s1, (int)(last - first - 1));
    const uint32_t a0 = b0 & ~15u;
    const bool staged = b1 - a0 <= kQ13SliceBytes;
    if (staged) {
      // Up to kQ13StageBatch 16-byte loads per lane in flight, then the stores.
      for (uint32_t base = (uint32_t)lane * 16u; a0 + base < b1; base += kQ13StageBatch * 512u) {
        uint4 v[kQ13StageBatch];
#pragma unroll
        for (int k = 0; k < kQ13StageBatch; ++k) {
          const uint32_t off = base + (uint32_t)k * 512u;
          if (a0 + off < b1 && a0 + off + 16u <= total)
            v[k] = __ldg(reinterpret_cast<const uint4*>(data + a0 + off));
        }
#pragma unroll
        for (int k = 0; k < kQ13StageBatch; ++k) {
          const uint32_t off = base + (uint32_t)k * 512u;
          if (a0 + off < b1) {
            if (a0 + off + 16u <= total) {
              *reinterpret_cast<uint4*>(slice + off) = v[k];
            } else {
              for (uint32_t j = 0; a0 + off + j < total; ++j) slice[off + j] = __ldg(data + a0 + off + j);
            }
          }
        }
      }
    }
    __syncwarp();
    if (i < last) {
      const bool hit = staged ? q13_match_slice(slice, (int)(s0 - a0), (int)(s1 - s0), w1, (int)l1, w2, (int)l2)
                              : q13_match(data + s0, s1 - s0, w1, l1, w2, l2);
      if (!hit) {
        if (c < 0 || (int64_t)c >= n_counts) {
          raise_error(err, kErrValueRange);
        } else {
          local_max = max(local_max, atomicAdd(counts + c, 1u) + 1u);
        }
      }
    }
    __syncwarp();
  }
  for (int o = 16; o; o >>= 1) local_max = max(local_max, __shfl_xor_sync(0xffffffffu, local_max, o));
  if (lane == 0 && local_max) atomicMax(max_count, local_max);
}

__global__ void __launch_bounds__(kQ13Block) q13_customer_kernel(const int32_t* __restrict__ c_custkey, int64_t n,
                                                                 const uint32_t* __restrict__ counts,
                                                                 int64_t n_counts, uint32_t* __restrict__ dist,
                                                                 uint32_t* err) {
  __shared__ uint32_t hist[kQ13SmallBins];
  for (int b = threadIdx.x; b < kQ13SmallBins; b += kQ13Block) hist[b] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * kQ13Block + threadIdx.x; i < n; i += (int64_t)gridDim.x * kQ13Block) {
    const int32_t c = c_custkey[i];
    if (c < 0 || (int64_t)c >= n_counts) {
      raise_error(err, kErrValueRange);
      continue;
    }
    const uint32_t cnt = counts[c];
    if (cnt < (uint32_t)kQ13SmallBins)
      atomicAdd(hist + cnt, 1u);
    else
      atomicAdd(dist + cnt, 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kQ13SmallBins; b += kQ13Block)
    if (hist[b]) atomicAdd(dist + b, hist[b]);
}

// Bins [0, *max_count] -> (key, c_count); each bin is cleared as it is read.
__global__ void __launch_bounds__(kQ13Block) q13_emit_kernel(uint32_t* __restrict__ dist,
                                                             const uint32_t* __restrict__ max_count,
                                                             unsigned long long* __restrict__ keys,
                                                             uint32_t* __restrict__ vals, unsigned long long* n_out) {
  __shared__ uint32_t warp_off[kQ13Warps];
  __shared__ unsigned long long base;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t bins = (int64_t)*max_count + 1;
  for (int64_t b0 = (int64_t)blockIdx.x * kQ13Block; b0 < bins; b0 += (int64_t)gridDim.x * kQ13Block) {
    const int64_t c = b0 + threadIdx.x;
    uint32_t v = 0;
    if (c < bins) {
      v = dist[c];
      if (v) dist[c] = 0;
    }
    const bool keep = v != 0;
    const uint32_t m = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) warp_off[warp] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t t = 0;
      for (int w = 0; w < kQ13Warps; ++w) {
        const uint32_t x = warp_off[w];
        warp_off[w] = t;
        t += x;
      }
      base = t ? atomicAdd(n_out, (unsigned long long)t) : 0ull;
    }
    __syncthreads();
    if (keep) {
      const unsigned long long pos = base + warp_off[warp] + __popc(m & ((1u << lane) - 1u));
      keys[pos] = ((unsigned long long)(0xffffffffu - v) << 32) | (0xffffffffu - (uint32_t)c);
      vals[pos] = (uint32_t)c;
    }
    __syncthreads();
  }
}

__global__ void q13_gather_kernel(const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ vals,
                                  const unsigned long long* n_out, uint32_t* max_count,
                                  bo_tpch_q13_row* __restrict__ out) {
  const unsigned long long n = *n_out;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    out[i].c_count = (int64_t)vals[i];
    out[i].custdist = (int64_t)(0xffffffffu - (uint32_t)(keys[i] >> 32));
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *max_count = 0;  // the emit kernel has read it
}

int q13_grid(bo_ctx* ctx, int64_t items) {
  const int64_t need = (items + kQ13Block - 1) / kQ13Block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)ctx->num_sms * 8));
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q13(bo_ctx* ctx, const bo_tpch_q13_tables* t, const char* word1, int64_t len1,
                           const char* word2, int64_t len2, bo_tpch_q13_row* out_host, int64_t max_rows,
                           int64_t* n_rows) {
  BO_CHECK_CTX(ctx);
  if (!t || !n_rows || max_rows < 0 || (max_rows > 0 && !out_host) || len1 < 0 || len2 < 0 ||
      (len1 > 0 && !word1) || (len2 > 0 && !word2))
    return set_error(ctx, BO_ERR_INVALID, "q13: null argument");
  if (t->n_orders < 0 || t->n_customer < 0 || t->n_count_map < 0)
    return set_error(ctx, BO_ERR_INVALID, "q13: negative size");
  if (t->n_orders >= 0xffffffffll || t->n_count_map > 0x80000000ll || len1 + len2 > 0x7fffffffll)
    return set_error(ctx, BO_ERR_INVALID, "q13: sizes beyond 32-bit counts");
  if ((t->n_orders > 0 && (!t->o_custkey || !t->o_comment_offsets || !t->o_comment)) ||
      (t->n_customer > 0 && !t->c_custkey))
    return set_error(ctx, BO_ERR_INVALID, "q13: null column");
  if (reinterpret_cast<uintptr_t>(t->o_comment) & 15u)
    return set_error(ctx, BO_ERR_INVALID, "q13: comment bytes must be 16-byte aligned");
  *n_rows = 0;
  if (t->n_customer == 0) return BO_OK;
  const int64_t no = t->n_orders, nm = std::max<int64_t>(t->n_count_map, 1);
  const int64_t n_dist = no + 1;  // an order count is at most n_orders
  const size_t wbytes = (size_t)(len1 + len2);
  // The histogram and the largest count live in their own region, all zero
  // between calls: zero-filled when (re)allocated, and each call's emit /
  // gather kernels clear exactly the bins and the count it set.
  void* hp = nullptr;
  int rc = region(ctx, "q13_hist", 256 + 4 * (size_t)n_dist, &hp);
  if (rc) return rc;
  auto* max_count = static_cast<uint32_t*>(hp);
  auto* dist = reinterpret_cast<uint32_t*>(static_cast<char*>(hp) + 256);
  size_t total = 0;
  auto add = [&](size_t b) { total += (b + 255) & ~size_t(255); };
  add(4 * (size_t)nm);      // counts per custkey
  add(8 * (size_t)n_dist);  // keys
  add(4 * (size_t)n_dist);  // vals
  add(8 * (size_t)n_dist);  // tmp keys
  add(4 * (size_t)n_dist);  // tmp vals
  add(sizeof(bo_tpch_q13_row) * (size_t)n_dist);
  add(64);                  // row count
  add(std::max<size_t>(wbytes, 1));
  void* basep = nullptr;
  if ((rc = region(ctx, "q13_ws", total, &basep))) return rc;
  char* p = static_cast<char*>(basep);
  auto* counts = carve<uint32_t>(p, (size_t)nm);
  auto* keys = carve<unsigned long long>(p, (size_t)n_dist);
  auto* vals = carve<uint32_t>(p, (size_t)n_dist);
  auto* tkeys = carve<unsigned long long>(p, (size_t)n_dist);
  auto* tvals = carve<uint32_t>(p, (size_t)n_dist);
  auto* rows = carve<bo_tpch_q13_row>(p, (size_t)n_dist);
  auto* n_out = carve<unsigned long long>(p, 8);
  auto* words = carve<uint8_t>(p, std::max<size_t>(wbytes, 1));
  if (wbytes) {
    void* h = nullptr;
    if ((rc = host_stage(ctx, wbytes, &h))) return rc;
    if (len1) std::memcpy(h, word1, (size_t)len1);
    if (len2) std::memcpy(static_cast<char*>(h) + len1, word2, (size_t)len2);
    BO_CUDA(ctx, cudaMemcpyAsync(words, h, wbytes, cudaMemcpyHostToDevice, ctx->stream));
  }
  BO_CUDA(ctx, cudaMemsetAsync(counts, 0, 4 * (size_t)nm, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(n_out, 0, 8, ctx->stream));
  // A failure after the histogram was written leaves it cleared for the next call.
  auto fail = [&](int code) {
    cudaMemsetAsync(hp, 0, 256 + 4 * (size_t)n_dist, ctx->stream);
    return code;
  };
  if (no > 0) {
    const int64_t groups = (no + 31) / 32;
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>((groups + kQ13Warps - 1) / kQ13Warps, (int64_t)ctx->num_sms * 6));
    q13_orders_kernel<<<grid, kQ13Block, 0, ctx->stream>>>(t->o_comment, t->o_comment_offsets, t->o_custkey, no,
                                                           words, (uint32_t)len1, (uint32_t)len2, counts,
                                                           t->n_count_map, max_count, ctx->d_err);
    if ((rc = after_launch(ctx, "q13_orders_kernel"))) return fail(rc);
  }
  q13_customer_kernel<<<q13_grid(ctx, t->n_customer), kQ13Block, 0, ctx->stream>>>(
      t->c_custkey, t->n_customer, counts, t->n_count_map, dist, ctx->d_err);
  if ((rc = after_launch(ctx, "q13_customer_kernel"))) return fail(rc);
  q13_emit_kernel<<<q13_grid(ctx, n_dist), kQ13Block, 0, ctx->stream>>>(dist, max_count, keys, vals, n_out);
  if ((rc = after_launch(ctx, "q13_emit_kernel"))) return fail(rc);
  if ((rc = radix_sort_pairs(ctx, keys, vals, tkeys, tvals, n_dist, 0, 64, n_out))) return fail(rc);
  q13_gather_kernel<<<q13_grid(ctx, n_dist), kQ13Block, 0, ctx->stream>>>(keys, vals, n_out, max_count, rows);
  if ((rc = after_launch(ctx, "q13_gather_kernel"))) return fail(rc);
  unsigned long long n = 0;
  BO_CUDA(ctx, cudaMemcpyAsync(&n, n_out, 8, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // synchronises the stream
  if ((rc = device_error_status(ctx, bits, "q13"))) return rc;
  *n_rows = (int64_t)n;
  const int64_t m = std::min<int64_t>((int64_t)n, max_rows);
  if (m > 0) {
    BO_CUDA(ctx, cudaMemcpyAsync(out_host, rows, sizeof(bo_tpch_q13_row) * (size_t)m, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return BO_OK;
}
