// TPC-H Q15 over the storage-plan layout: run_q15 of
// bespoke_tpch/query_q15.cpp:215-534.
//
// The reference sums the discounted price per supplier over the lineitem
// shards of the quarter (whole months outside the window are skipped, which
// drops nothing the date test would keep), then returns the suppliers whose
// total equals the largest.  Here one lineitem pass: eight shipdates per
// 16-byte load; rows in the window read suppkey and price and add to a
// per-block shared total for suppkeys below 4096 (larger ones straight to
// the global totals); the maximum and the supplier rows are taken on the
// host from the per-suppkey totals.
#include <algorithm>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ15Block = 256;
constexpr int kQ15Rows = 8;
constexpr int kQ15SmallKeys = 4096;

__global__ void __launch_bounds__(kQ15Block) q15_kernel(bo_tpch_q15_tables t, int64_t n_supp, int32_t start,
                                                        uint32_t span, unsigned long long* __restrict__ revenue,
                                                        unsigned long long* __restrict__ shipped) {
  __shared__ unsigned long long acc[kQ15SmallKeys];
  const int small = n_supp < kQ15SmallKeys ? (int)n_supp : kQ15SmallKeys;
  for (int i = threadIdx.x; i < small; i += kQ15Block) acc[i] = 0;
  __syncthreads();
  unsigned long long count = 0;
  const int64_t stride = (int64_t)gridDim.x * kQ15Block;
  for (int64_t g = (int64_t)blockIdx.x * kQ15Block + threadIdx.x; g * kQ15Rows < t.n_lineitem; g += stride) {
    const int64_t r0 = g * kQ15Rows;
    int32_t sd[kQ15Rows];
    uint32_t valid = 0xffu;
    if (r0 + kQ15Rows <= t.n_lineitem) {
      const int4 s4 = ld_stream_v4(t.l_shipdate + r0);
      const uint32_t sw[4] = {(uint32_t)s4.x, (uint32_t)s4.y, (uint32_t)s4.z, (uint32_t)s4.w};
#pragma unroll
      for (int k = 0; k < kQ15Rows; ++k) sd[k] = (int32_t)(int16_t)((sw[k >> 1] >> (16 * (k & 1))) & 0xffffu);
    } else {
      valid = 0;
#pragma unroll
      for (int k = 0; k < kQ15Rows; ++k) {
        sd[k] = 0;
        if (r0 + k < t.n_lineitem) {
          sd[k] = t.l_shipdate[r0 + k];
          valid |= 1u << k;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kQ15Rows; ++k) {
      if (!((valid >> k) & 1u) || (uint32_t)(sd[k] - start) >= span) continue;
      ++count;
      const int32_t sk = t.l_suppkey[r0 + k];
      if (sk < 0 || (int64_t)sk >= n_supp) continue;
      const unsigned long long v = (unsigned long long)(long long)t.l_discounted_price[r0 + k];
      if (sk < small)
        atomicAdd(acc + sk, v);
      else
        atomicAdd(revenue + sk, v);
    }
  }
  for (int o = 16; o; o >>= 1) count += __shfl_xor_sync(0xffffffffu, count, o);
  if ((threadIdx.x & 31) == 0 && count) atomicAdd(shipped, count);
  __syncthreads();
  for (int i = threadIdx.x; i < small; i += kQ15Block)
    if (acc[i]) atomicAdd(revenue + i, acc[i]);
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q15(bo_ctx* ctx, const bo_tpch_q15_tables* t, int64_t n_supp, int16_t start_offset,
                           int16_t end_offset, int64_t* revenue_out, int64_t* shipped_out) {
  BO_CHECK_CTX(ctx);
  if (!t || !shipped_out || (n_supp > 0 && !revenue_out)) return set_error(ctx, BO_ERR_INVALID, "q15: null argument");
  if (t->n_lineitem < 0 || n_supp < 0) return set_error(ctx, BO_ERR_INVALID, "q15: negative size");
  if (t->n_lineitem > 0 && (!t->l_shipdate || !t->l_suppkey || !t->l_discounted_price))
    return set_error(ctx, BO_ERR_INVALID, "q15: null column");
  if (t->n_lineitem > 0 && !aligned16(t->l_shipdate))
    return set_error(ctx, BO_ERR_INVALID, "q15: shipdates must be 16-byte aligned");
  for (int64_t i = 0; i < n_supp; ++i) revenue_out[i] = 0;
  *shipped_out = 0;
  if (t->n_lineitem == 0) return BO_OK;
  const size_t bytes = 256 + sizeof(unsigned long long) * (size_t)std::max<int64_t>(n_supp, 1);
  void* p = nullptr;
  int rc = region(ctx, "q15_ws", bytes, &p);
  if (rc) return rc;
  auto* shipped = static_cast<unsigned long long*>(p);
  auto* revenue = shipped + 32;
  BO_CUDA(ctx, cudaMemsetAsync(p, 0, bytes, ctx->stream));
  const int64_t groups = (t->n_lineitem + kQ15Rows - 1) / kQ15Rows;
  const int64_t resident =
      (int64_t)ctx->num_sms * occupancy_blocks(reinterpret_cast<const void*>(&q15_kernel), kQ15Block, 0);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((groups + kQ15Block - 1) / kQ15Block, resident));
  q15_kernel<<<grid, kQ15Block, 0, ctx->stream>>>(*t, n_supp, start_offset,
                                                  (uint32_t)((int32_t)end_offset - (int32_t)start_offset), revenue,
                                                  shipped);
  if ((rc = after_launch(ctx, "q15_kernel"))) return rc;
  unsigned long long s = 0;
  BO_CUDA(ctx, cudaMemcpyAsync(&s, shipped, 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (n_supp > 0)
    BO_CUDA(ctx, cudaMemcpyAsync(revenue_out, revenue, sizeof(int64_t) * (size_t)n_supp, cudaMemcpyDeviceToHost,
                                 ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *shipped_out = (int64_t)s;
  return BO_OK;
}
