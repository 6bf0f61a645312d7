// TPC-H Q12 over the storage-plan layout: run_q12 of
// bespoke_tpch/query_q12.cpp:162-360.
//
// The reference walks the lineitem shards that can hold a receipt in the
// date window, keeps lineitems of the two ship modes with shipdate <
// commitdate < receiptdate and receiptdate in the window, looks up each
// one's order through orderkey_to_row and counts it as high or low by the
// order's priority.  Here one pass over lineitem: each thread takes eight
// consecutive rows (16-byte loads of the shipmode codes and shipdates, a
// 32-byte load of the packed commit / receipt dates), tests them in
// registers, and only the few survivors read their orderkey, order row and
// priority.  Four counters (high / low for each of the two modes) per
// thread, reduced per warp and per block, one 64-bit atomic each per block.
// The shard pruning is kept exactly through the optional per-lineitem
// latest shipdate of its shard (computed by the builder when some lineitem
// could be pruned at all).
#include <algorithm>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ12Block = 256;
constexpr int kQ12Rows = 8;
constexpr int32_t kReceiptLagMaxDays = 30;  // query_q12.cpp:178

struct Q12Args {
  const uint16_t* mode;
  const uint32_t* cr;
  const int16_t* ship;
  const int32_t* okey;
  const int16_t* shard_max;
  int64_t n;
  const int32_t* map;
  int64_t n_map;
  const uint16_t* prio;
  int64_t n_orders;
  int32_t c1, c2, h1, h2;
  int32_t start, ship_min;
  uint32_t span;
};

__global__ void __launch_bounds__(kQ12Block) q12_kernel(Q12Args a, unsigned long long* __restrict__ counts,
                                                        uint32_t* err) {
  uint32_t c[4] = {0, 0, 0, 0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g * kQ12Rows < a.n; g += stride) {
    const int64_t r0 = g * kQ12Rows;
    uint32_t md[kQ12Rows], cr[kQ12Rows];
    int32_t sd[kQ12Rows];
    uint32_t valid = 0xffu;
    if (r0 + kQ12Rows <= a.n) {
      const int4 m4 = ld_stream_v4(a.mode + r0);
      const int4 s4 = ld_stream_v4(a.ship + r0);
      const int8v c8 = ld_stream_v8(a.cr + r0);
      const uint32_t mw[4] = {(uint32_t)m4.x, (uint32_t)m4.y, (uint32_t)m4.z, (uint32_t)m4.w};
      const uint32_t sw[4] = {(uint32_t)s4.x, (uint32_t)s4.y, (uint32_t)s4.z, (uint32_t)s4.w};
#pragma unroll
      for (int k = 0; k < kQ12Rows; ++k) {
        md[k] = (mw[k >> 1] >> (16 * (k & 1))) & 0xffffu;
        sd[k] = (int32_t)(int16_t)((sw[k >> 1] >> (16 * (k & 1))) & 0xffffu);
        cr[k] = (uint32_t)c8.v[k];
      }
    } else {
      valid = 0;
#pragma unroll
      for (int k = 0; k < kQ12Rows; ++k) {
        md[k] = 0;
        sd[k] = 0;
        cr[k] = 0;
        if (r0 + k < a.n) {
          md[k] = a.mode[r0 + k];
          sd[k] = a.ship[r0 + k];
          cr[k] = a.cr[r0 + k];
          valid |= 1u << k;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kQ12Rows; ++k) {
      const int32_t m = (int32_t)md[k];
      if (!((valid >> k) & 1u) || (m != a.c1 && m != a.c2)) continue;
      const int32_t commit = (int32_t)(int16_t)(cr[k] & 0xffffu);
      const int32_t receipt = (int32_t)(int16_t)(cr[k] >> 16);
      if (commit >= receipt || sd[k] >= commit) continue;
      if ((uint32_t)(receipt - a.start) >= a.span) continue;
      if (a.shard_max && (int32_t)a.shard_max[r0 + k] < a.ship_min) continue;
      const int32_t ok = a.okey[r0 + k];
      if ((uint64_t)(uint32_t)ok >= (uint64_t)a.n_map) continue;
      const int32_t row = a.map[ok];
      if (row < 0) continue;
      if ((int64_t)row >= a.n_orders) {  // the reference would read past its orders
        raise_error(err, kErrValueRange);
        continue;
      }
      const int32_t pc = (int32_t)a.prio[row];
      const bool high = pc == a.h1 || pc == a.h2;
      ++c[(m == a.c1 ? 0 : 2) + (high ? 0 : 1)];
    }
  }
  __shared__ unsigned long long part[4][kQ12Block / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    unsigned long long v = c[i];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) part[i][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    unsigned long long t = 0;
    for (int w = 0; w < kQ12Block / 32; ++w) t += part[threadIdx.x][w];
    if (t) atomicAdd(counts + threadIdx.x, t);
  }
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q12(bo_ctx* ctx, const bo_tpch_q12_tables* t, int32_t mode_code1, int32_t mode_code2,
                           int32_t high_code1, int32_t high_code2, int16_t start_offset, int16_t end_offset,
                           int64_t counts_out[4]) {
  BO_CHECK_CTX(ctx);
  if (!t || !counts_out) return set_error(ctx, BO_ERR_INVALID, "q12: null argument");
  if (t->n_lineitem < 0 || t->n_orderkey_map < 0 || t->n_orders < 0)
    return set_error(ctx, BO_ERR_INVALID, "q12: negative size");
  if ((t->n_lineitem > 0 && (!t->l_shipmode || !t->l_commit_receipt || !t->l_shipdate || !t->l_orderkey)) ||
      (t->n_orderkey_map > 0 && !t->orderkey_to_row) || (t->n_orders > 0 && !t->o_orderpriority))
    return set_error(ctx, BO_ERR_INVALID, "q12: null column");
  if (t->n_lineitem > 0 && (!aligned16(t->l_shipmode) || !aligned16(t->l_shipdate) ||
                            !aligned32(t->l_commit_receipt)))
    return set_error(ctx, BO_ERR_INVALID, "q12: lineitem columns must be 16-byte (commit_receipt 32-byte) aligned");
  for (int i = 0; i < 4; ++i) counts_out[i] = 0;
  if (t->n_lineitem == 0 || (mode_code1 < 0 && mode_code2 < 0)) return BO_OK;
  void* p = nullptr;
  int rc = region(ctx, "q12_counts", 64, &p);
  if (rc) return rc;
  auto* counts = static_cast<unsigned long long*>(p);
  BO_CUDA(ctx, cudaMemsetAsync(counts, 0, 4 * sizeof(unsigned long long), ctx->stream));
  Q12Args a;
  a.mode = t->l_shipmode;
  a.cr = t->l_commit_receipt;
  a.ship = t->l_shipdate;
  a.okey = t->l_orderkey;
  a.shard_max = t->l_shard_max_shipdate;
  a.n = t->n_lineitem;
  a.map = t->orderkey_to_row;
  a.n_map = t->n_orderkey_map;
  a.prio = t->o_orderpriority;
  a.n_orders = t->n_orders;
  a.c1 = mode_code1;
  a.c2 = mode_code2;
  a.h1 = high_code1;
  a.h2 = high_code2;
  a.start = start_offset;
  a.ship_min = (int32_t)start_offset - kReceiptLagMaxDays;
  a.span = (uint32_t)((int32_t)end_offset - (int32_t)start_offset);
  const int64_t groups = (t->n_lineitem + kQ12Rows - 1) / kQ12Rows;
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(reinterpret_cast<const void*>(&q12_kernel),
                                                                    kQ12Block, 0);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((groups + kQ12Block - 1) / kQ12Block, resident));
  q12_kernel<<<grid, kQ12Block, 0, ctx->stream>>>(a, counts, ctx->d_err);
  if ((rc = after_launch(ctx, "q12_kernel"))) return rc;
  unsigned long long h[4];
  BO_CUDA(ctx, cudaMemcpyAsync(h, counts, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // synchronises the stream
  if ((rc = device_error_status(ctx, bits, "q12"))) return rc;
  for (int i = 0; i < 4; ++i) counts_out[i] = (int64_t)h[i];
  return BO_OK;
}
