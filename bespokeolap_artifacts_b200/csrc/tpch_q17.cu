// TPC-H Q17 over the storage-plan layout: run_q17 of
// bespoke_tpch/query_q17.cpp:119-311.
//
// The reference marks the parts of one brand and container in a bitmap,
// scans lineitem once to total quantity and count per marked part while
// keeping the matching rows, then sums the extended price of the kept rows
// whose quantity is below a fifth of their part's average.  Here:
//   parts   one thread per part row sets its bit (atomicOr);
//   scan    eight lineitems per thread (one 32-byte partkey load); the few
//           marked ones add to their part's sum and count and append their
//           row to a list (one reservation per warp);
//   filter  one thread per listed row tests 5 * qty * count < sum; an int64
//           block sum, one atomic per block.
#include <algorithm>

#include "common.cuh"
#include "context.cuh"
#include "rows.cuh"

namespace bo {
namespace {

constexpr int kQ17Block = 256;
constexpr int kQ17Rows = 8;

__global__ void __launch_bounds__(kQ17Block) q17_part_kernel(const int32_t* __restrict__ key,
                                                             const uint16_t* __restrict__ brand,
                                                             const uint16_t* __restrict__ container, int64_t n,
                                                             int32_t max_key, int32_t b, int32_t c,
                                                             uint32_t* __restrict__ bits) {
  for (int64_t i = (int64_t)blockIdx.x * kQ17Block + threadIdx.x; i < n; i += (int64_t)gridDim.x * kQ17Block) {
    const int32_t k = key[i];
    if (k < 0 || k > max_key) continue;
    if ((int32_t)brand[i] == b && (int32_t)container[i] == c) atomicOr(bits + (k >> 5), 1u << (k & 31));
  }
}

__global__ void __launch_bounds__(kQ17Block) q17_scan_kernel(const int32_t* __restrict__ partkey,
                                                             const int16_t* __restrict__ qty, int64_t n,
                                                             uint32_t max_key, const uint32_t* __restrict__ bits,
                                                             unsigned long long* __restrict__ sum,
                                                             uint32_t* __restrict__ cnt, uint32_t* __restrict__ list,
                                                             unsigned long long* __restrict__ n_list) {
  const int lane = threadIdx.x & 31;
  const int64_t groups = (n + kQ17Rows - 1) / kQ17Rows;
  const int64_t groups_w = (groups + 31) & ~int64_t(31);  // whole warps iterate together
  for (int64_t g = (int64_t)blockIdx.x * kQ17Block + threadIdx.x; g < groups_w;
       g += (int64_t)gridDim.x * kQ17Block) {
    const int64_t r0 = g * kQ17Rows;
    uint32_t pk[kQ17Rows];
    uint32_t hit = 0;
    if (r0 + kQ17Rows <= n) {
      const int8v v = ld_stream_v8(partkey + r0);
#pragma unroll
      for (int k = 0; k < kQ17Rows; ++k) pk[k] = (uint32_t)v.v[k];
    } else {
#pragma unroll
      for (int k = 0; k < kQ17Rows; ++k) pk[k] = r0 + k < n ? (uint32_t)partkey[r0 + k] : 0xffffffffu;
    }
#pragma unroll
    for (int k = 0; k < kQ17Rows; ++k)
      if (pk[k] <= max_key && ((__ldg(bits + (pk[k] >> 5)) >> (pk[k] & 31)) & 1u)) hit |= 1u << k;
    const uint32_t mine = __popc(hit);
    uint32_t total;
    uint32_t pos = warp_exclusive_scan(mine, total);
    if (total == 0) continue;  // warp-uniform
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(n_list, (unsigned long long)total);
    base = __shfl_sync(0xffffffffu, base, 0);
#pragma unroll
    for (int k = 0; k < kQ17Rows; ++k) {
      if (!((hit >> k) & 1u)) continue;
      const int64_t row = r0 + k;
      atomicAdd(sum + pk[k], (unsigned long long)(long long)qty[row]);
      atomicAdd(cnt + pk[k], 1u);
      list[base + pos++] = (uint32_t)row;
    }
  }
}

__global__ void __launch_bounds__(kQ17Block) q17_filter_kernel(const uint32_t* __restrict__ list,
                                                               const unsigned long long* __restrict__ n_list,
                                                               const int32_t* __restrict__ partkey,
                                                               const int16_t* __restrict__ qty,
                                                               const int32_t* __restrict__ price,
                                                               const unsigned long long* __restrict__ sum,
                                                               const uint32_t* __restrict__ cnt,
                                                               unsigned long long* __restrict__ out) {
  const unsigned long long m = *n_list;
  long long acc = 0;
  for (unsigned long long i = (unsigned long long)blockIdx.x * kQ17Block + threadIdx.x; i < m;
       i += (unsigned long long)gridDim.x * kQ17Block) {
    const uint32_t row = list[i];
    const uint32_t pk = (uint32_t)partkey[row];
    const long long c = (long long)cnt[pk];
    const long long lhs = (long long)qty[row] * 5 * c;  // query_q17.cpp:290-295
    if (lhs < (long long)sum[pk]) acc += price[row];
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ long long part[kQ17Block / 32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int w = 0; w < kQ17Block / 32; ++w) s += part[w];
    if (s) atomicAdd(out, (unsigned long long)s);
  }
}

int q17_grid(bo_ctx* ctx, int64_t items) {
  const int64_t need = (items + kQ17Block - 1) / kQ17Block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)ctx->num_sms * 8));
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q17(bo_ctx* ctx, const bo_tpch_q17_tables* t, int32_t brand_code, int32_t container_code,
                           int64_t* sum_out) {
  BO_CHECK_CTX(ctx);
  if (!t || !sum_out) return set_error(ctx, BO_ERR_INVALID, "q17: null argument");
  if (t->n_lineitem < 0 || t->n_part < 0) return set_error(ctx, BO_ERR_INVALID, "q17: negative size");
  if (t->n_lineitem > 0xffffffffll) return set_error(ctx, BO_ERR_INVALID, "q17: more than 2^32 lineitems");
  if ((t->n_lineitem > 0 && (!t->l_partkey || !t->l_quantity || !t->l_extendedprice)) ||
      (t->n_part > 0 && (!t->p_partkey || !t->p_brand || !t->p_container)))
    return set_error(ctx, BO_ERR_INVALID, "q17: null column");
  if (t->n_lineitem > 0 && !aligned32(t->l_partkey))
    return set_error(ctx, BO_ERR_INVALID, "q17: partkeys must be 32-byte aligned");
  *sum_out = 0;
  if (t->max_partkey < 0 || t->n_part == 0 || t->n_lineitem == 0 || brand_code < 0 || container_code < 0)
    return BO_OK;
  const int64_t keys = (int64_t)t->max_partkey + 1;
  const int64_t words = (keys + 31) / 32;
  size_t total = 0;
  auto add = [&](size_t b) { total += (b + 255) & ~size_t(255); };
  add(4 * (size_t)words);
  add(8 * (size_t)keys);
  add(4 * (size_t)keys);
  add(4 * (size_t)t->n_lineitem);
  add(64);
  void* base = nullptr;
  int rc = region(ctx, "q17_ws", total, &base);
  if (rc) return rc;
  char* p = static_cast<char*>(base);
  auto* bits = carve<uint32_t>(p, (size_t)words);
  auto* sum = carve<unsigned long long>(p, (size_t)keys);
  auto* cnt = carve<uint32_t>(p, (size_t)keys);
  auto* list = carve<uint32_t>(p, (size_t)t->n_lineitem);
  auto* ctr = carve<unsigned long long>(p, 8);  // [0] list length, [1] result
  BO_CUDA(ctx, cudaMemsetAsync(bits, 0, 4 * (size_t)words, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(sum, 0, 8 * (size_t)keys, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(cnt, 0, 4 * (size_t)keys, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(ctr, 0, 16, ctx->stream));
  q17_part_kernel<<<q17_grid(ctx, t->n_part), kQ17Block, 0, ctx->stream>>>(
      t->p_partkey, t->p_brand, t->p_container, t->n_part, t->max_partkey, brand_code, container_code, bits);
  if ((rc = after_launch(ctx, "q17_part_kernel"))) return rc;
  q17_scan_kernel<<<q17_grid(ctx, (t->n_lineitem + kQ17Rows - 1) / kQ17Rows), kQ17Block, 0, ctx->stream>>>(
      t->l_partkey, t->l_quantity, t->n_lineitem, (uint32_t)t->max_partkey, bits, sum, cnt, list, ctr);
  if ((rc = after_launch(ctx, "q17_scan_kernel"))) return rc;
  q17_filter_kernel<<<q17_grid(ctx, std::min<int64_t>(t->n_lineitem, (int64_t)ctx->num_sms * 8 * kQ17Block)),
                      kQ17Block, 0, ctx->stream>>>(list, ctr, t->l_partkey, t->l_quantity, t->l_extendedprice, sum,
                                                   cnt, ctr + 1);
  if ((rc = after_launch(ctx, "q17_filter_kernel"))) return rc;
  unsigned long long r = 0;
  BO_CUDA(ctx, cudaMemcpyAsync(&r, ctr + 1, 8, cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *sum_out = (int64_t)r;
  return BO_OK;
}
