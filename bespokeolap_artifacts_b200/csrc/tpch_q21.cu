// TPC-H Q21 over the storage-plan layout: run_q21 of
// bespoke_tpch/query_q21.cpp:145-392.
//
// The reference walks the lineitem range of every order with the final
// status: an order counts for supplier s when its lineitems name more than
// one supplier and s is the only supplier with late lineitems (receipt after
// commit); s's wait count grows by those lineitems when s is of the nation.
// Here one thread per order walks its range (stopping at a second late
// supplier, as the reference does) and adds its count with one 64-bit atomic
// per counting order; the supplier rows and the ordering are taken on the
// host from the per-suppkey counts.
#include <algorithm>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ21Block = 256;

template <bool kSorted>
__global__ void __launch_bounds__(kQ21Block) q21_orders_kernel(bo_tpch_q21_tables t, uint32_t final_code,
                                                               uint32_t max_suppkey,
                                                               const uint8_t* __restrict__ target,
                                                               unsigned long long* __restrict__ waits, uint32_t* err) {
  const int64_t stride = (int64_t)gridDim.x * kQ21Block;
  for (int64_t i = (int64_t)blockIdx.x * kQ21Block + threadIdx.x; i < t.n_orders; i += stride) {
    if (t.o_orderstatus[i] != final_code) continue;
    const uint32_t e = t.o_li_end[i];
    if (e == 0u) continue;
    const uint32_t b = t.o_li_begin[i];
    if ((int64_t)e > t.n_lineitem || b > e) {  // a range that is not one of this lineitem table's
      raise_error(err, kErrValueRange);
      continue;
    }
    if (e - b <= 1u) continue;
    const int32_t key = kSorted ? 0 : t.o_orderkey[i];
    int32_t first = -1, late_supp = -1;
    uint32_t late_n = 0;
    bool multi = false, multi_late = false;
    for (uint32_t j = b; j < e; ++j) {
      if (!kSorted && t.l_orderkey[j] != key) continue;
      const int32_t sk = t.l_suppkey[j];
      if ((uint32_t)sk > max_suppkey) continue;
      if (first < 0)
        first = sk;
      else if (sk != first)
        multi = true;
      const uint32_t cr = t.l_commit_receipt[j];
      if ((cr >> 16) > (cr & 0xffffu)) {
        if (late_supp == -1 || late_supp == sk) {
          late_supp = sk;
          ++late_n;
        } else {
          multi_late = true;
          break;
        }
      }
    }
    if (multi_late || !multi || late_supp < 0 || !target[late_supp]) continue;
    atomicAdd(waits + late_supp, (unsigned long long)late_n);
  }
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q21(bo_ctx* ctx, const bo_tpch_q21_tables* t, int32_t final_code, const uint8_t* target_host,
                           int32_t max_suppkey, int64_t* waits_out) {
  BO_CHECK_CTX(ctx);
  if (!t || max_suppkey < 0 || !target_host || !waits_out)
    return set_error(ctx, BO_ERR_INVALID, "q21: null argument or negative supplier key bound");
  if (t->n_orders < 0 || t->n_lineitem < 0 || final_code < 0)
    return set_error(ctx, BO_ERR_INVALID, "q21: negative size or status code");
  const size_t n_keys = (size_t)max_suppkey + 1;
  for (size_t i = 0; i < n_keys; ++i) waits_out[i] = 0;
  if (t->n_orders == 0 || t->n_lineitem == 0) return BO_OK;
  if (!t->o_orderstatus || !t->o_li_begin || !t->o_li_end || !t->l_suppkey || !t->l_commit_receipt ||
      (!t->lineitem_orderkey_sorted && (!t->o_orderkey || !t->l_orderkey)))
    return set_error(ctx, BO_ERR_INVALID, "q21: null column");
  const size_t wait_bytes = (sizeof(unsigned long long) * n_keys + 255) & ~size_t(255);
  void* p = nullptr;
  int rc = region(ctx, "q21_ws", wait_bytes + n_keys, &p);
  if (rc) return rc;
  auto* waits = static_cast<unsigned long long*>(p);
  auto* target = static_cast<uint8_t*>(p) + wait_bytes;
  BO_CUDA(ctx, cudaMemsetAsync(waits, 0, wait_bytes, ctx->stream));
  BO_CUDA(ctx, cudaMemcpyAsync(target, target_host, n_keys, cudaMemcpyHostToDevice, ctx->stream));
  const int64_t resident = (int64_t)ctx->num_sms *
                           occupancy_blocks(reinterpret_cast<const void*>(&q21_orders_kernel<true>), kQ21Block, 0);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((t->n_orders + kQ21Block - 1) / kQ21Block, resident));
  if (t->lineitem_orderkey_sorted)
    q21_orders_kernel<true><<<grid, kQ21Block, 0, ctx->stream>>>(*t, (uint32_t)final_code, (uint32_t)max_suppkey,
                                                                  target, waits, ctx->d_err);
  else
    q21_orders_kernel<false><<<grid, kQ21Block, 0, ctx->stream>>>(*t, (uint32_t)final_code, (uint32_t)max_suppkey,
                                                                   target, waits, ctx->d_err);
  if ((rc = after_launch(ctx, "q21_orders_kernel"))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(waits_out, waits, sizeof(int64_t) * n_keys, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // synchronises the stream
  return device_error_status(ctx, bits, "q21");
}
