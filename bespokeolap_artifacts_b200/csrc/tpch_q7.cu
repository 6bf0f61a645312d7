// TPC-H Q7 over the storage-plan layout: run_q7 of
// bespoke_tpch/query_q7.cpp:140-435.
//
// The reference tags suppliers of the two nations, then (lineitems sorted by
// orderkey) walks the lineitem ranges of the orders whose customer is in one
// of them, or (otherwise) scans lineitem and finds each one's order through
// orderkey_to_row; both sum the discounted price of lineitems shipped in
// 1995-1996 by (supplier nation, customer nation, year).  Both give the same
// sums, so here one lineitem pass serves both layouts: eight shipdates per
// 16-byte load; rows in the window read their suppkey and the tag (a small
// table), tagged ones their order's customer nation.  Eight int64 sums per
// thread, reduced per warp and per block.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ7Block = 256;
constexpr int kQ7Rows = 8;

struct Q7Args {
  bo_tpch_q7_tables t;
  const int8_t* tag;
  int64_t n_tag;
  int32_t nation1, nation2, start, span, year2;
  bool same;
};

__global__ void __launch_bounds__(kQ7Block) q7_kernel(Q7Args a, unsigned long long* __restrict__ revenue) {
  long long acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const bo_tpch_q7_tables& t = a.t;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g * kQ7Rows < t.n_lineitem; g += stride) {
    const int64_t r0 = g * kQ7Rows;
    int32_t sd[kQ7Rows];
    uint32_t valid = 0xffu;
    if (r0 + kQ7Rows <= t.n_lineitem) {
      const int4 s4 = ld_stream_v4(t.l_shipdate + r0);
      const uint32_t sw[4] = {(uint32_t)s4.x, (uint32_t)s4.y, (uint32_t)s4.z, (uint32_t)s4.w};
#pragma unroll
      for (int k = 0; k < kQ7Rows; ++k) sd[k] = (int32_t)(int16_t)((sw[k >> 1] >> (16 * (k & 1))) & 0xffffu);
    } else {
      valid = 0;
#pragma unroll
      for (int k = 0; k < kQ7Rows; ++k) {
        sd[k] = 0;
        if (r0 + k < t.n_lineitem) {
          sd[k] = t.l_shipdate[r0 + k];
          valid |= 1u << k;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kQ7Rows; ++k) {
      if (!((valid >> k) & 1u) || (uint32_t)(sd[k] - a.start) > (uint32_t)a.span) continue;
      const int32_t sk = t.l_suppkey[r0 + k];
      if (sk < 0 || (int64_t)sk >= a.n_tag) continue;
      const int32_t supp = a.tag[sk];
      if (supp < 0) continue;
      const int32_t ok = t.l_orderkey[r0 + k];
      if (ok < 0 || (int64_t)ok >= t.n_orderkey_map) continue;
      const int32_t row = t.orderkey_to_row[ok];
      if (row < 0 || (int64_t)row >= t.n_orders) continue;
      const int32_t cn = t.o_cust_nation[row];
      int32_t cust;
      if (cn == a.nation1)
        cust = 0;
      else if (!a.same && cn == a.nation2)
        cust = 1;
      else
        continue;
      if (a.same ? (supp != 0 || cust != 0) : supp == cust) continue;
      acc[supp * 4 + cust * 2 + (sd[k] >= a.year2 ? 1 : 0)] += t.l_discounted_price[r0 + k];
    }
  }
  __shared__ long long part[8][kQ7Block / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    long long v = acc[i];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) part[i][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    long long s = 0;
    for (int w = 0; w < kQ7Block / 32; ++w) s += part[threadIdx.x][w];
    if (s) atomicAdd(revenue + threadIdx.x, (unsigned long long)s);
  }
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q7(bo_ctx* ctx, const bo_tpch_q7_tables* t, const int8_t* supp_tag_host, int64_t n_supp_tag,
                          int32_t nation1, int32_t nation2, int16_t ship_start, int16_t ship_last,
                          int16_t year2_start, int64_t revenue_out[8]) {
  BO_CHECK_CTX(ctx);
  if (!t || !revenue_out || (n_supp_tag > 0 && !supp_tag_host))
    return set_error(ctx, BO_ERR_INVALID, "q7: null argument");
  if (t->n_lineitem < 0 || t->n_orderkey_map < 0 || t->n_orders < 0 || n_supp_tag < 0)
    return set_error(ctx, BO_ERR_INVALID, "q7: negative size");
  if ((t->n_lineitem > 0 && (!t->l_shipdate || !t->l_suppkey || !t->l_orderkey || !t->l_discounted_price)) ||
      (t->n_orderkey_map > 0 && !t->orderkey_to_row) || (t->n_orders > 0 && !t->o_cust_nation))
    return set_error(ctx, BO_ERR_INVALID, "q7: null column");
  if (t->n_lineitem > 0 && !aligned16(t->l_shipdate))
    return set_error(ctx, BO_ERR_INVALID, "q7: shipdates must be 16-byte aligned");
  for (int i = 0; i < 8; ++i) revenue_out[i] = 0;
  if (t->n_lineitem == 0 || n_supp_tag == 0) return BO_OK;
  const size_t tag_bytes = ((size_t)n_supp_tag + 255) & ~size_t(255);
  void* p = nullptr;
  int rc = region(ctx, "q7_ws", 256 + tag_bytes, &p);
  if (rc) return rc;
  auto* revenue = static_cast<unsigned long long*>(p);
  auto* tag = static_cast<int8_t*>(p) + 256;
  void* h = nullptr;
  if ((rc = host_stage(ctx, (size_t)n_supp_tag, &h))) return rc;
  std::memcpy(h, supp_tag_host, (size_t)n_supp_tag);
  BO_CUDA(ctx, cudaMemcpyAsync(tag, h, (size_t)n_supp_tag, cudaMemcpyHostToDevice, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(revenue, 0, 8 * sizeof(unsigned long long), ctx->stream));
  Q7Args a;
  a.t = *t;
  a.tag = tag;
  a.n_tag = n_supp_tag;
  a.nation1 = nation1;
  a.nation2 = nation2;
  a.start = ship_start;
  a.span = (int32_t)ship_last - (int32_t)ship_start;
  a.year2 = year2_start;
  a.same = nation1 == nation2;
  const int64_t groups = (t->n_lineitem + kQ7Rows - 1) / kQ7Rows;
  const int64_t resident =
      (int64_t)ctx->num_sms * occupancy_blocks(reinterpret_cast<const void*>(&q7_kernel), kQ7Block, 0);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((groups + kQ7Block - 1) / kQ7Block, resident));
  q7_kernel<<<grid, kQ7Block, 0, ctx->stream>>>(a, revenue);
  if ((rc = after_launch(ctx, "q7_kernel"))) return rc;
  unsigned long long hv[8];
  BO_CUDA(ctx, cudaMemcpyAsync(hv, revenue, sizeof(hv), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < 8; ++i) revenue_out[i] = (int64_t)hv[i];
  return BO_OK;
}
