// TPC-H Q4 over the storage-plan layout: run_q4 of
// bespoke_tpch/query_q4.cpp:172-355.
//
// The reference takes the date-sorted orders of a three-month window, walks
// each order's lineitem range until a lineitem with commit < receipt, and
// counts the orders that have one by priority.  Here one thread per order of
// the window (the window's rows found by the same test on the sorted dates),
// its range walked with early exit; counts per priority code gathered in a
// per-block shared histogram (codes below 1024; larger codes straight to the
// global counts), one atomic per non-zero bin per block.
#include <algorithm>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ4Block = 256;
constexpr int kQ4SmallCodes = 1024;

template <bool kSorted>
__global__ void __launch_bounds__(kQ4Block) q4_orders_kernel(bo_tpch_q4_tables t, int16_t start, int16_t end,
                                                             unsigned long long* __restrict__ counts, uint32_t* err) {
  __shared__ uint32_t hist[kQ4SmallCodes];
  for (int i = threadIdx.x; i < kQ4SmallCodes; i += kQ4Block) hist[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * kQ4Block + threadIdx.x; i < t.n_orders; i += (int64_t)gridDim.x * kQ4Block) {
    const int16_t d = t.o_orderdate[i];
    if (d < start || d >= end) continue;
    const uint32_t e = t.o_li_end[i];
    if (e == 0u) continue;
    const uint32_t b = t.o_li_begin[i];
    if ((int64_t)e > t.n_lineitem || b > e) {  // a range that is not one of this lineitem table's
      raise_error(err, kErrValueRange);
      continue;
    }
    const int32_t key = kSorted ? 0 : t.o_orderkey[i];
    bool late = false;
    for (uint32_t j = b; j < e && !late; ++j) {
      if (!kSorted && t.l_orderkey[j] != key) continue;
      const uint32_t cr = t.l_commit_receipt[j];
      late = (uint16_t)cr < (uint16_t)(cr >> 16);
    }
    if (!late) continue;
    const uint32_t code = t.o_orderpriority[i];
    if (code >= (uint32_t)t.n_priorities) {
      raise_error(err, kErrValueRange);
      continue;
    }
    if (code < (uint32_t)kQ4SmallCodes)
      atomicAdd(hist + code, 1u);
    else
      atomicAdd(counts + code, 1ull);
  }
  __syncthreads();
  const int lim = min(t.n_priorities, kQ4SmallCodes);
  for (int c = threadIdx.x; c < lim; c += kQ4Block)
    if (hist[c]) atomicAdd(counts + c, (unsigned long long)hist[c]);
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q4(bo_ctx* ctx, const bo_tpch_q4_tables* t, int16_t start_offset, int16_t end_offset,
                          int64_t* counts_out) {
  BO_CHECK_CTX(ctx);
  if (!t || (t->n_priorities > 0 && !counts_out)) return set_error(ctx, BO_ERR_INVALID, "q4: null argument");
  if (t->n_orders < 0 || t->n_lineitem < 0 || t->n_priorities < 0)
    return set_error(ctx, BO_ERR_INVALID, "q4: negative size");
  if (t->n_priorities > 65536) return set_error(ctx, BO_ERR_INVALID, "q4: more than 65536 priority codes");
  if ((t->n_orders > 0 && (!t->o_orderkey || !t->o_orderdate || !t->o_orderpriority || !t->o_li_begin ||
                           !t->o_li_end)) ||
      (t->n_lineitem > 0 && (!t->l_orderkey || !t->l_commit_receipt)))
    return set_error(ctx, BO_ERR_INVALID, "q4: null column");
  for (int32_t i = 0; i < t->n_priorities; ++i) counts_out[i] = 0;
  if (t->n_orders == 0 || t->n_lineitem == 0 || t->n_priorities == 0) return BO_OK;
  void* p = nullptr;
  const size_t bytes = sizeof(unsigned long long) * (size_t)t->n_priorities;
  int rc = region(ctx, "q4_counts", bytes, &p);
  if (rc) return rc;
  auto* counts = static_cast<unsigned long long*>(p);
  BO_CUDA(ctx, cudaMemsetAsync(counts, 0, bytes, ctx->stream));
  const int64_t resident = (int64_t)ctx->num_sms *
                           occupancy_blocks(reinterpret_cast<const void*>(&q4_orders_kernel<true>), kQ4Block, 0);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((t->n_orders + kQ4Block - 1) / kQ4Block, resident));
  if (t->lineitem_orderkey_sorted)
    q4_orders_kernel<true><<<grid, kQ4Block, 0, ctx->stream>>>(*t, start_offset, end_offset, counts, ctx->d_err);
  else
    q4_orders_kernel<false><<<grid, kQ4Block, 0, ctx->stream>>>(*t, start_offset, end_offset, counts, ctx->d_err);
  if ((rc = after_launch(ctx, "q4_orders_kernel"))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(counts_out, counts, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // synchronises the stream
  return device_error_status(ctx, bits, "q4");
}
