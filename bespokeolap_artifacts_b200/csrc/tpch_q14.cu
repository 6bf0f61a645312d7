// TPC-H Q14 over the storage-plan layout: run_q14 of
// bespoke_tpch/query_q14.cpp:176-352.
//
// The reference walks the lineitem shards that overlap the month and sums
// the discounted price of each lineitem shipped in it whose part exists,
// separately for parts of a PROMO type.  Here one pass over lineitem: each
// thread tests eight shipdates from one 16-byte load; only the rows in the
// month (about one in eighty over seven years of dates) read their partkey,
// price and the part's promo flag (a one-byte-per-partkey table that stays
// in L2).  Two int64 sums per thread, reduced per warp and per block, one
// 64-bit atomic each per block.
#include <algorithm>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ14Block = 256;
constexpr int kQ14Rows = 8;

__global__ void __launch_bounds__(kQ14Block) q14_kernel(bo_tpch_q14_tables t, int32_t start, int32_t end,
                                                        unsigned long long* __restrict__ sums) {
  long long promo = 0, total = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g * kQ14Rows < t.n_lineitem; g += stride) {
    const int64_t r0 = g * kQ14Rows;
    int32_t sd[kQ14Rows];
    uint32_t valid = 0xffu;
    if (r0 + kQ14Rows <= t.n_lineitem) {
      const int4 s4 = ld_stream_v4(t.l_shipdate + r0);
      const uint32_t sw[4] = {(uint32_t)s4.x, (uint32_t)s4.y, (uint32_t)s4.z, (uint32_t)s4.w};
#pragma unroll
      for (int k = 0; k < kQ14Rows; ++k) sd[k] = (int32_t)(int16_t)((sw[k >> 1] >> (16 * (k & 1))) & 0xffffu);
    } else {
      valid = 0;
#pragma unroll
      for (int k = 0; k < kQ14Rows; ++k) {
        sd[k] = 0;
        if (r0 + k < t.n_lineitem) {
          sd[k] = t.l_shipdate[r0 + k];
          valid |= 1u << k;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kQ14Rows; ++k) {
      if (!((valid >> k) & 1u) || sd[k] < start || sd[k] >= end) continue;
      const int32_t key = t.l_partkey[r0 + k];
      if (key < 0 || (int64_t)key >= t.n_promo_map) continue;
      const int8_t flag = t.p_promo_by_key[key];
      if (flag < 0) continue;
      const long long price = t.l_discounted_price[r0 + k];
      total += price;
      if (flag) promo += price;
    }
  }
  __shared__ long long part[2][kQ14Block / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o; o >>= 1) {
    promo += __shfl_xor_sync(0xffffffffu, promo, o);
    total += __shfl_xor_sync(0xffffffffu, total, o);
  }
  if (lane == 0) {
    part[0][warp] = promo;
    part[1][warp] = total;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    long long s = 0;
    for (int w = 0; w < kQ14Block / 32; ++w) s += part[threadIdx.x][w];
    if (s) atomicAdd(sums + threadIdx.x, (unsigned long long)s);  // two's complement: signed sums add exactly
  }
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q14(bo_ctx* ctx, const bo_tpch_q14_tables* t, int16_t start_offset, int16_t end_offset,
                           int64_t sums_out[2]) {
  BO_CHECK_CTX(ctx);
  if (!t || !sums_out) return set_error(ctx, BO_ERR_INVALID, "q14: null argument");
  if (t->n_lineitem < 0 || t->n_promo_map < 0) return set_error(ctx, BO_ERR_INVALID, "q14: negative size");
  if ((t->n_lineitem > 0 && (!t->l_shipdate || !t->l_partkey || !t->l_discounted_price)) ||
      (t->n_promo_map > 0 && !t->p_promo_by_key))
    return set_error(ctx, BO_ERR_INVALID, "q14: null column");
  if (t->n_lineitem > 0 && !aligned16(t->l_shipdate))
    return set_error(ctx, BO_ERR_INVALID, "q14: shipdates must be 16-byte aligned");
  sums_out[0] = sums_out[1] = 0;
  if (t->n_lineitem == 0 || t->n_promo_map == 0) return BO_OK;
  void* p = nullptr;
  int rc = region(ctx, "q14_sums", 64, &p);
  if (rc) return rc;
  auto* sums = static_cast<unsigned long long*>(p);
  BO_CUDA(ctx, cudaMemsetAsync(sums, 0, 2 * sizeof(unsigned long long), ctx->stream));
  const int64_t groups = (t->n_lineitem + kQ14Rows - 1) / kQ14Rows;
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(reinterpret_cast<const void*>(&q14_kernel),
                                                                    kQ14Block, 0);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((groups + kQ14Block - 1) / kQ14Block, resident));
  q14_kernel<<<grid, kQ14Block, 0, ctx->stream>>>(*t, start_offset, end_offset, sums);
  if ((rc = after_launch(ctx, "q14_kernel"))) return rc;
  unsigned long long h[2];
  BO_CUDA(ctx, cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  sums_out[0] = (int64_t)h[0];
  sums_out[1] = (int64_t)h[1];
  return BO_OK;
}
