// TPC-H Q5 over the storage-plan layout: run_q5 of
// bespoke_tpch/query_q5.cpp:197-540.
//
// The reference takes the date-sorted orders of a one-year window, keeps
// those whose customer's nation lies in the region, and sums over each
// order's lineitem range the discounted prices of lineitems supplied from
// that same nation.  Both nations are precomputed per row by the builder
// (orders' customer nation, lineitems' supplier nation), so the query is a
// range walk: one thread per order of the window, revenue per nation
// gathered in a per-block shared array (nations below 256; larger keys
// straight to the global sums), one 64-bit atomic per non-zero nation per
// block.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ5Block = 256;
constexpr int kQ5SmallNations = 256;

template <bool kSorted>
__global__ void __launch_bounds__(kQ5Block) q5_orders_kernel(bo_tpch_q5_tables t, const uint8_t* __restrict__ in_region,
                                                             int16_t start, int16_t end,
                                                             unsigned long long* __restrict__ revenue, uint32_t* err) {
  __shared__ unsigned long long acc[kQ5SmallNations];
  for (int i = threadIdx.x; i < kQ5SmallNations; i += kQ5Block) acc[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * kQ5Block + threadIdx.x; i < t.n_orders; i += (int64_t)gridDim.x * kQ5Block) {
    const int16_t d = t.o_orderdate[i];
    if (d < start || d >= end) continue;
    const int32_t cn = t.o_cust_nation[i];
    if (cn < 0 || cn >= t.n_nations || !in_region[cn]) continue;
    const uint32_t e = t.o_li_end[i];
    if (e == 0u) continue;
    const uint32_t b = t.o_li_begin[i];
    if ((int64_t)e > t.n_lineitem || b > e) {  // a range that is not one of this lineitem table's
      raise_error(err, kErrValueRange);
      continue;
    }
    const int32_t key = kSorted ? 0 : t.o_orderkey[i];
    unsigned long long rev = 0;  // int64 sum, wrapping as the reference's
    for (uint32_t j = b; j < e; ++j) {
      if (!kSorted && t.l_orderkey[j] != key) continue;
      if ((int32_t)t.l_supp_nation[j] != cn) continue;
      rev += (unsigned long long)(long long)t.l_discounted_price[j];
    }
    if (rev == 0ull) continue;
    if (cn < kQ5SmallNations)
      atomicAdd(acc + cn, rev);
    else
      atomicAdd(revenue + cn, rev);
  }
  __syncthreads();
  const int lim = min(t.n_nations, kQ5SmallNations);
  for (int c = threadIdx.x; c < lim; c += kQ5Block)
    if (acc[c]) atomicAdd(revenue + c, acc[c]);
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q5(bo_ctx* ctx, const bo_tpch_q5_tables* t, const uint8_t* nation_in_region_host,
                          int16_t start_offset, int16_t end_offset, int64_t* revenue_out) {
  BO_CHECK_CTX(ctx);
  if (!t || (t->n_nations > 0 && (!revenue_out || !nation_in_region_host)))
    return set_error(ctx, BO_ERR_INVALID, "q5: null argument");
  if (t->n_orders < 0 || t->n_lineitem < 0 || t->n_nations < 0)
    return set_error(ctx, BO_ERR_INVALID, "q5: negative size");
  if (t->n_nations > 32768) return set_error(ctx, BO_ERR_INVALID, "q5: nation keys beyond int16");
  if ((t->n_orders > 0 && (!t->o_orderkey || !t->o_orderdate || !t->o_cust_nation || !t->o_li_begin ||
                           !t->o_li_end)) ||
      (t->n_lineitem > 0 && (!t->l_orderkey || !t->l_supp_nation || !t->l_discounted_price)))
    return set_error(ctx, BO_ERR_INVALID, "q5: null column");
  for (int32_t i = 0; i < t->n_nations; ++i) revenue_out[i] = 0;
  if (t->n_orders == 0 || t->n_lineitem == 0 || t->n_nations == 0) return BO_OK;
  const size_t sums = sizeof(unsigned long long) * (size_t)t->n_nations;
  const size_t mask = ((size_t)t->n_nations + 255) & ~size_t(255);
  void* p = nullptr;
  int rc = region(ctx, "q5_ws", sums + mask, &p);
  if (rc) return rc;
  auto* revenue = static_cast<unsigned long long*>(p);
  auto* in_region = static_cast<uint8_t*>(p) + sums;
  void* h = nullptr;
  if ((rc = host_stage(ctx, (size_t)t->n_nations, &h))) return rc;
  std::memcpy(h, nation_in_region_host, (size_t)t->n_nations);
  BO_CUDA(ctx, cudaMemcpyAsync(in_region, h, (size_t)t->n_nations, cudaMemcpyHostToDevice, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(revenue, 0, sums, ctx->stream));
  const int64_t resident = (int64_t)ctx->num_sms *
                           occupancy_blocks(reinterpret_cast<const void*>(&q5_orders_kernel<true>), kQ5Block, 0);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((t->n_orders + kQ5Block - 1) / kQ5Block, resident));
  if (t->lineitem_orderkey_sorted)
    q5_orders_kernel<true><<<grid, kQ5Block, 0, ctx->stream>>>(*t, in_region, start_offset, end_offset, revenue,
                                                               ctx->d_err);
  else
    q5_orders_kernel<false><<<grid, kQ5Block, 0, ctx->stream>>>(*t, in_region, start_offset, end_offset, revenue,
                                                                ctx->d_err);
  if ((rc = after_launch(ctx, "q5_orders_kernel"))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(revenue_out, revenue, sums, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // synchronises the stream
  return device_error_status(ctx, bits, "q5");
}
