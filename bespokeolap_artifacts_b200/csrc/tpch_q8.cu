// TPC-H Q8 over the storage-plan layout: run_q8 of
// bespoke_tpch/query_q8.cpp:122-380.
//
// The reference marks the custkeys whose customer lies in the region, the
// suppkeys of the target nation and the partkeys of the type, then (sorted
// lineitems) walks the lineitem ranges of the window's orders of marked
// customers, or (otherwise) marks qualifying orderkeys and scans lineitem;
// both add each qualifying lineitem's volume to its order year's total, and
// to the nation's share when its supplier is marked.  For orderkeys that
// are unique the two forms agree, and one lineitem pass serves both here:
//   marks    one thread per customer / part row sets its key's byte;
//   scan     eight lineitems per thread (one 32-byte partkey load); marked
//            parts read their order (key -> row -> date, custkey) and, when
//            it qualifies, price, discount and the supplier mark.
// Four int64 sums per thread, reduced per warp and per block.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ8Block = 256;
constexpr int kQ8Rows = 8;

__global__ void __launch_bounds__(kQ8Block) q8_mark_kernel(const int32_t* __restrict__ c_key,
                                                           const int32_t* __restrict__ c_nation, int64_t n_cust,
                                                           int32_t max_custkey, const uint8_t* __restrict__ in_region,
                                                           int32_t n_nations, uint8_t* __restrict__ cust_ok,
                                                           const int32_t* __restrict__ p_key,
                                                           const uint16_t* __restrict__ p_type, int64_t n_part,
                                                           int32_t max_partkey, int32_t type_code,
                                                           uint8_t* __restrict__ part_ok) {
  const int64_t stride = (int64_t)gridDim.x * kQ8Block;
  for (int64_t i = (int64_t)blockIdx.x * kQ8Block + threadIdx.x; i < n_cust; i += stride) {
    const int32_t k = c_key[i], nk = c_nation[i];
    if (k < 0 || k > max_custkey || nk < 0 || nk >= n_nations) continue;
    if (in_region[nk]) cust_ok[k] = 1;
  }
  for (int64_t i = (int64_t)blockIdx.x * kQ8Block + threadIdx.x; i < n_part; i += stride) {
    const int32_t k = p_key[i];
    if (k < 0 || k > max_partkey) continue;
    if ((int32_t)p_type[i] == type_code) part_ok[k] = 1;
  }
}

struct Q8Args {
  bo_tpch_q8_tables t;
  const uint8_t* cust_ok;
  const uint8_t* part_ok;
  const uint8_t* supp;
  int64_t n_supp;
  int32_t start, span, year2;
};

__global__ void __launch_bounds__(kQ8Block) q8_scan_kernel(Q8Args a, unsigned long long* __restrict__ sums) {
  const bo_tpch_q8_tables& t = a.t;
  long long nation[2] = {0, 0}, total[2] = {0, 0};
  const int64_t stride = (int64_t)gridDim.x * kQ8Block;
  for (int64_t g = (int64_t)blockIdx.x * kQ8Block + threadIdx.x; g * kQ8Rows < t.n_lineitem; g += stride) {
    const int64_t r0 = g * kQ8Rows;
    int32_t pk[kQ8Rows];
    if (r0 + kQ8Rows <= t.n_lineitem) {
      const int8v v = ld_stream_v8(t.l_partkey + r0);
#pragma unroll
      for (int k = 0; k < kQ8Rows; ++k) pk[k] = v.v[k];
    } else {
#pragma unroll
      for (int k = 0; k < kQ8Rows; ++k) pk[k] = r0 + k < t.n_lineitem ? t.l_partkey[r0 + k] : -1;
    }
#pragma unroll
    for (int k = 0; k < kQ8Rows; ++k) {
      if (pk[k] < 0 || pk[k] > t.max_partkey || !a.part_ok[pk[k]]) continue;
      const int64_t r = r0 + k;
      const int32_t ok = t.l_orderkey[r];
      if (ok < 0 || (int64_t)ok >= t.n_orderkey_map) continue;
      const int32_t row = t.orderkey_to_row[ok];
      if (row < 0 || (int64_t)row >= t.n_orders) continue;
      const int32_t d = t.o_orderdate[row];
      if ((uint32_t)(d - a.start) > (uint32_t)a.span) continue;
      const int32_t ck = t.o_custkey[row];
      if (ck < 0 || ck > t.max_custkey || !a.cust_ok[ck]) continue;
      const long long volume = (long long)t.l_extendedprice[r] * (100 - (int32_t)t.l_discount[r]);
      const int y = d >= a.year2 ? 1 : 0;
      total[y] += volume;
      const int32_t sk = t.l_suppkey[r];
      if (sk >= 0 && (int64_t)sk < a.n_supp && a.supp[sk]) nation[y] += volume;
    }
  }
  __shared__ long long part[4][kQ8Block / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  long long v[4] = {nation[0], nation[1], total[0], total[1]};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    for (int o = 16; o; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
    if (lane == 0) part[i][warp] = v[i];
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    long long s = 0;
    for (int w = 0; w < kQ8Block / 32; ++w) s += part[threadIdx.x][w];
    if (s) atomicAdd(sums + threadIdx.x, (unsigned long long)s);
  }
}

int q8_grid(bo_ctx* ctx, int64_t items) {
  const int64_t need = (items + kQ8Block - 1) / kQ8Block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)ctx->num_sms * 8));
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q8(bo_ctx* ctx, const bo_tpch_q8_tables* t, const uint8_t* nation_in_region_host,
                          int32_t n_nations, const uint8_t* supp_target_host, int64_t n_supp, int32_t type_code,
                          int16_t date_start, int16_t date_last, int16_t year2_start, int64_t sums_out[4]) {
  BO_CHECK_CTX(ctx);
  if (!t || !sums_out || (n_nations > 0 && !nation_in_region_host) || (n_supp > 0 && !supp_target_host))
    return set_error(ctx, BO_ERR_INVALID, "q8: null argument");
  if (t->n_lineitem < 0 || t->n_orderkey_map < 0 || t->n_orders < 0 || t->n_customer < 0 || t->n_part < 0 ||
      n_nations < 0 || n_supp < 0)
    return set_error(ctx, BO_ERR_INVALID, "q8: negative size");
  if ((t->n_lineitem > 0 && (!t->l_partkey || !t->l_suppkey || !t->l_orderkey || !t->l_extendedprice ||
                             !t->l_discount)) ||
      (t->n_orderkey_map > 0 && !t->orderkey_to_row) || (t->n_orders > 0 && (!t->o_custkey || !t->o_orderdate)) ||
      (t->n_customer > 0 && (!t->c_custkey || !t->c_nationkey)) || (t->n_part > 0 && (!t->p_partkey || !t->p_type)))
    return set_error(ctx, BO_ERR_INVALID, "q8: null column");
  if (t->n_lineitem > 0 && !aligned32(t->l_partkey))
    return set_error(ctx, BO_ERR_INVALID, "q8: partkeys must be 32-byte aligned");
  for (int i = 0; i < 4; ++i) sums_out[i] = 0;
  if (t->n_lineitem == 0 || t->max_partkey < 0 || t->max_custkey < 0 || type_code < 0) return BO_OK;
  const size_t nc = (size_t)t->max_custkey + 1, np = (size_t)t->max_partkey + 1;
  size_t total = 0;
  auto add = [&](size_t b) { total += (b + 255) & ~size_t(255); };
  add(64);                                   // sums
  add(nc);                                   // custkey marks
  add(np);                                   // partkey marks
  add((size_t)std::max<int32_t>(n_nations, 1));
  add((size_t)std::max<int64_t>(n_supp, 1));
  void* base = nullptr;
  int rc = region(ctx, "q8_ws", total, &base);
  if (rc) return rc;
  char* p = static_cast<char*>(base);
  auto* sums = carve<unsigned long long>(p, 8);
  auto* cust_ok = carve<uint8_t>(p, nc);
  auto* part_ok = carve<uint8_t>(p, np);
  auto* in_region = carve<uint8_t>(p, (size_t)std::max<int32_t>(n_nations, 1));
  auto* supp = carve<uint8_t>(p, (size_t)std::max<int64_t>(n_supp, 1));
  const size_t hb = (size_t)n_nations + (size_t)n_supp;
  if (hb > 0) {
    void* h = nullptr;
    if ((rc = host_stage(ctx, hb, &h))) return rc;
    if (n_nations > 0) std::memcpy(h, nation_in_region_host, (size_t)n_nations);
    if (n_supp > 0) std::memcpy(static_cast<char*>(h) + n_nations, supp_target_host, (size_t)n_supp);
    if (n_nations > 0)
      BO_CUDA(ctx, cudaMemcpyAsync(in_region, h, (size_t)n_nations, cudaMemcpyHostToDevice, ctx->stream));
    if (n_supp > 0)
      BO_CUDA(ctx, cudaMemcpyAsync(supp, static_cast<char*>(h) + n_nations, (size_t)n_supp, cudaMemcpyHostToDevice,
                                   ctx->stream));
  }
  BO_CUDA(ctx, cudaMemsetAsync(sums, 0, 4 * sizeof(unsigned long long), ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(cust_ok, 0, nc, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(part_ok, 0, np, ctx->stream));
  q8_mark_kernel<<<q8_grid(ctx, std::max<int64_t>(t->n_customer, t->n_part)), kQ8Block, 0, ctx->stream>>>(
      t->c_custkey, t->c_nationkey, t->n_customer, t->max_custkey, in_region, n_nations, cust_ok, t->p_partkey,
      t->p_type, t->n_part, t->max_partkey, type_code, part_ok);
  if ((rc = after_launch(ctx, "q8_mark_kernel"))) return rc;
  Q8Args a;
  a.t = *t;
  a.cust_ok = cust_ok;
  a.part_ok = part_ok;
  a.supp = supp;
  a.n_supp = n_supp;
  a.start = date_start;
  a.span = (int32_t)date_last - (int32_t)date_start;
  a.year2 = year2_start;
  const int64_t groups = (t->n_lineitem + kQ8Rows - 1) / kQ8Rows;
  const int64_t resident =
      (int64_t)ctx->num_sms * occupancy_blocks(reinterpret_cast<const void*>(&q8_scan_kernel), kQ8Block, 0);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((groups + kQ8Block - 1) / kQ8Block, resident));
  q8_scan_kernel<<<grid, kQ8Block, 0, ctx->stream>>>(a, sums);
  if ((rc = after_launch(ctx, "q8_scan_kernel"))) return rc;
  unsigned long long hv[4];
  BO_CUDA(ctx, cudaMemcpyAsync(hv, sums, sizeof(hv), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < 4; ++i) sums_out[i] = (int64_t)hv[i];
  return BO_OK;
}
