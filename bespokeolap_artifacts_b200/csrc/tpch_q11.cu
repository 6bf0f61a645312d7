// TPC-H Q11 over the storage-plan layout: run_q11 of
// bespoke_tpch/query_q11.cpp:109-224.
//
// The reference walks partsupp (sorted by partkey by the builder) once,
// summing the stock value of the nation's suppliers per partkey run and in
// total; parts whose sum exceeds a fraction of the total are returned.
// Here one thread per partsupp row adds its value to its partkey's sum
// (each partkey is one run of the sorted rows, so per-key sums are the run
// sums) and to a per-block total; the threshold, the filter and the order
// are applied on the host to the per-key sums.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ11Block = 256;

__global__ void __launch_bounds__(kQ11Block) q11_kernel(bo_tpch_q11_tables t, const uint8_t* __restrict__ in_nation,
                                                        int64_t n_supp, unsigned long long* __restrict__ sums,
                                                        unsigned long long* __restrict__ total, uint32_t* err) {
  long long acc = 0;
  const int64_t range = (int64_t)t.max_partkey - t.min_partkey + 1;
  for (int64_t i = (int64_t)blockIdx.x * kQ11Block + threadIdx.x; i < t.n_partsupp;
       i += (int64_t)gridDim.x * kQ11Block) {
    const int32_t sk = t.ps_suppkey[i];
    if (sk < 0 || (int64_t)sk >= n_supp || !in_nation[sk]) continue;
    const int64_t slot = (int64_t)t.ps_partkey[i] - t.min_partkey;
    if (slot < 0 || slot >= range) {
      raise_error(err, kErrValueRange);
      continue;
    }
    const long long v = t.ps_value[i];
    acc += v;
    atomicAdd(sums + slot, (unsigned long long)v);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(total, (unsigned long long)acc);
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q11(bo_ctx* ctx, const bo_tpch_q11_tables* t, const uint8_t* supp_in_nation_host,
                           int64_t n_supp, int64_t* sums_out, int64_t* total_out) {
  BO_CHECK_CTX(ctx);
  if (!t || !total_out || (n_supp > 0 && !supp_in_nation_host)) return set_error(ctx, BO_ERR_INVALID, "q11: null argument");
  if (t->n_partsupp < 0 || n_supp < 0) return set_error(ctx, BO_ERR_INVALID, "q11: negative size");
  *total_out = 0;
  if (t->n_partsupp == 0) return BO_OK;
  if (t->max_partkey < t->min_partkey) return set_error(ctx, BO_ERR_INVALID, "q11: empty partkey range");
  if (!t->ps_partkey || !t->ps_suppkey || !t->ps_value || !sums_out)
    return set_error(ctx, BO_ERR_INVALID, "q11: null column");
  const int64_t range = (int64_t)t->max_partkey - t->min_partkey + 1;
  for (int64_t i = 0; i < range; ++i) sums_out[i] = 0;
  if (n_supp == 0) return BO_OK;
  const size_t sum_bytes = sizeof(unsigned long long) * (size_t)range;
  const size_t mask_bytes = ((size_t)n_supp + 255) & ~size_t(255);
  void* p = nullptr;
  int rc = region(ctx, "q11_ws", 256 + sum_bytes + mask_bytes, &p);
  if (rc) return rc;
  auto* total = static_cast<unsigned long long*>(p);
  auto* sums = total + 32;
  auto* in_nation = reinterpret_cast<uint8_t*>(sums + range);
  void* h = nullptr;
  if ((rc = host_stage(ctx, (size_t)n_supp, &h))) return rc;
  std::memcpy(h, supp_in_nation_host, (size_t)n_supp);
  BO_CUDA(ctx, cudaMemcpyAsync(in_nation, h, (size_t)n_supp, cudaMemcpyHostToDevice, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(p, 0, 256 + sum_bytes, ctx->stream));
  const int64_t need = (t->n_partsupp + kQ11Block - 1) / kQ11Block;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)ctx->num_sms * 8));
  q11_kernel<<<grid, kQ11Block, 0, ctx->stream>>>(*t, in_nation, n_supp, sums, total, ctx->d_err);
  if ((rc = after_launch(ctx, "q11_kernel"))) return rc;
  unsigned long long tv = 0;
  BO_CUDA(ctx, cudaMemcpyAsync(&tv, total, 8, cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaMemcpyAsync(sums_out, sums, sum_bytes, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // synchronises the stream
  if ((rc = device_error_status(ctx, bits, "q11"))) return rc;
  *total_out = (int64_t)tv;
  return BO_OK;
}
