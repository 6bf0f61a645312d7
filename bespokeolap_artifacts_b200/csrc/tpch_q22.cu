// TPC-H Q22 over the storage-plan layout: run_q22 of
// bespoke_tpch/query_q22.cpp:272-540.
//
// The reference filters customers by phone prefix class and positive
// balance to get the average balance, then counts, per class, the
// customers above that average without orders (an empty range in the
// builder's orders-by-customer offsets).  Here two passes over customer:
//   stats  balance sum and count of the allowed positive balances;
//   emit   each block derives the integer average from those totals, keeps
//          the allowed customers above it whose custkey has no order bit,
//          and adds them to a per-block shared histogram of classes.
// The per-custkey order bits are built once by the drop-in's build().
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ22Block = 256;
constexpr int kQ22Classes = 100 + BO_Q22_MAX_EXTRA;

struct Q22Filter {
  uint8_t numeric[100];
  uint16_t extra[BO_Q22_MAX_EXTRA];
  int32_t n_extra;
};

// The customer's class (numeric code, or 100 + extra index) when allowed, else -1.
__device__ __forceinline__ int q22_class(const Q22Filter& f, uint8_t prefix, uint32_t pair) {
  if (prefix != 255u) return prefix < 100u && f.numeric[prefix] ? (int)prefix : -1;
  if (!(pair & 0x10000u)) return -1;
  for (int i = 0; i < f.n_extra; ++i)
    if ((uint32_t)f.extra[i] == (pair & 0xffffu)) return 100 + i;
  return -1;
}

__global__ void __launch_bounds__(kQ22Block) q22_stats_kernel(bo_tpch_q22_tables t, Q22Filter f,
                                                              unsigned long long* __restrict__ stats) {
  long long sum = 0, cnt = 0;
  for (int64_t i = (int64_t)blockIdx.x * kQ22Block + threadIdx.x; i < t.n_customer;
       i += (int64_t)gridDim.x * kQ22Block) {
    const int32_t bal = t.c_acctbal[i];
    if (bal <= 0 || q22_class(f, t.c_phone_prefix[i], t.c_phone_pair[i]) < 0) continue;
    sum += bal;
    ++cnt;
  }
  for (int o = 16; o; o >>= 1) {
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  }
  __shared__ long long part[2][kQ22Block / 32];
  if ((threadIdx.x & 31) == 0) {
    part[0][threadIdx.x >> 5] = sum;
    part[1][threadIdx.x >> 5] = cnt;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    long long s = 0;
    for (int w = 0; w < kQ22Block / 32; ++w) s += part[threadIdx.x][w];
    if (s) atomicAdd(stats + threadIdx.x, (unsigned long long)s);
  }
}

__global__ void __launch_bounds__(kQ22Block) q22_emit_kernel(bo_tpch_q22_tables t, Q22Filter f,
                                                             const unsigned long long* __restrict__ stats,
                                                             unsigned long long* __restrict__ out) {
  __shared__ unsigned long long h_cnt[kQ22Classes], h_sum[kQ22Classes];
  for (int i = threadIdx.x; i < kQ22Classes; i += kQ22Block) h_cnt[i] = h_sum[i] = 0;
  __syncthreads();
  const long long count = (long long)stats[1];
  if (count > 0) {
    const long long avg = (long long)stats[0] / count;  // query_q22.cpp:345, 455
    for (int64_t i = (int64_t)blockIdx.x * kQ22Block + threadIdx.x; i < t.n_customer;
         i += (int64_t)gridDim.x * kQ22Block) {
      const int32_t bal = t.c_acctbal[i];
      if (bal <= 0 || (long long)bal <= avg) continue;
      const int c = q22_class(f, t.c_phone_prefix[i], t.c_phone_pair[i]);
      if (c < 0) continue;
      const int32_t key = t.c_custkey[i];
      if (key >= 0 && (int64_t)key < t.n_order_custkeys && ((t.o_has_order[key >> 5] >> (key & 31)) & 1u)) continue;
      atomicAdd(h_cnt + c, 1ull);
      atomicAdd(h_sum + c, (unsigned long long)(long long)bal);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kQ22Classes; i += kQ22Block)
    if (h_cnt[i]) {
      atomicAdd(out + i, h_cnt[i]);
      atomicAdd(out + kQ22Classes + i, h_sum[i]);
    }
}

int q22_grid(bo_ctx* ctx, int64_t items) {
  const int64_t need = (items + kQ22Block - 1) / kQ22Block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)ctx->num_sms * 4));
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q22(bo_ctx* ctx, const bo_tpch_q22_tables* t, const uint8_t numeric_allowed[100],
                           const uint16_t* extra_pairs, int32_t n_extra, int64_t counts_out[107],
                           int64_t sums_out[107]) {
  BO_CHECK_CTX(ctx);
  if (!t || !numeric_allowed || !counts_out || !sums_out || (n_extra > 0 && !extra_pairs))
    return set_error(ctx, BO_ERR_INVALID, "q22: null argument");
  if (n_extra < 0 || n_extra > BO_Q22_MAX_EXTRA) return set_error(ctx, BO_ERR_INVALID, "q22: 0..7 extra prefixes");
  if (t->n_customer < 0 || t->n_order_custkeys < 0) return set_error(ctx, BO_ERR_INVALID, "q22: negative size");
  if ((t->n_customer > 0 && (!t->c_custkey || !t->c_acctbal || !t->c_phone_prefix || !t->c_phone_pair)) ||
      (t->n_order_custkeys > 0 && !t->o_has_order))
    return set_error(ctx, BO_ERR_INVALID, "q22: null column");
  for (int i = 0; i < kQ22Classes; ++i) counts_out[i] = sums_out[i] = 0;
  if (t->n_customer == 0) return BO_OK;
  Q22Filter f;
  std::memcpy(f.numeric, numeric_allowed, 100);
  for (int i = 0; i < BO_Q22_MAX_EXTRA; ++i) f.extra[i] = i < n_extra ? extra_pairs[i] : 0;
  f.n_extra = n_extra;
  void* p = nullptr;
  int rc = region(ctx, "q22_ws", 256 + 2 * kQ22Classes * sizeof(unsigned long long), &p);
  if (rc) return rc;
  auto* stats = static_cast<unsigned long long*>(p);
  auto* out = stats + 32;
  BO_CUDA(ctx, cudaMemsetAsync(p, 0, 256 + 2 * kQ22Classes * sizeof(unsigned long long), ctx->stream));
  const int grid = q22_grid(ctx, t->n_customer);
  q22_stats_kernel<<<grid, kQ22Block, 0, ctx->stream>>>(*t, f, stats);
  if ((rc = after_launch(ctx, "q22_stats_kernel"))) return rc;
  q22_emit_kernel<<<grid, kQ22Block, 0, ctx->stream>>>(*t, f, stats, out);
  if ((rc = after_launch(ctx, "q22_emit_kernel"))) return rc;
  unsigned long long hv[2 * kQ22Classes];
  BO_CUDA(ctx, cudaMemcpyAsync(hv, out, sizeof(hv), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < kQ22Classes; ++i) {
    counts_out[i] = (int64_t)hv[i];
    sums_out[i] = (int64_t)hv[kQ22Classes + i];
  }
  return BO_OK;
}
