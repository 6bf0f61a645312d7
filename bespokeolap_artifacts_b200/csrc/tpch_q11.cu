// TPC-H Q11 over the storage-plan layout: run_q11 of
// bespoke_tpch/query_q11.cpp:109-224.
//
// The reference walks partsupp (sorted by partkey by the builder) once,
// summing the stock value of the nation's suppliers per partkey run and in
// total; parts whose sum exceeds a fraction of the total are returned.
// Here one thread per partsupp row adds its value to its partkey's sum
// (each partkey is one run of the sorted rows, so per-key sums are the run
// sums) and to a per-block total; the threshold, the filter and the order
// are applied on the host to the per-key sums (bo_tpch_q11), or on the
// device (bo_tpch_q11_rows): an ordered compaction of the keys above the
// threshold (ascending partkey) and one stable sort by value descending.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "compact.cuh"
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

// :186-195: a non-zero sum above total * FRACTION (compared as doubles).
struct Q11Kept {
  const unsigned long long* sums;
  const unsigned long long* total;
  double fraction;
  __device__ __forceinline__ bool operator()(int64_t i, uint32_t& v) const {
    const long long s = (long long)__ldg(sums + i);
    if (s == 0) return false;
    const double threshold = (double)(long long)__ldg(total) * fraction;
    if (!((double)s > threshold)) return false;
    v = (uint32_t)i;
    return true;
  }
};

// The first min(*n_dev, limit) entries.
__device__ __forceinline__ int64_t q11_count(const unsigned long long* n_dev, int64_t limit) {
  const unsigned long long nd = *n_dev;
  return nd < (unsigned long long)limit ? (int64_t)nd : limit;
}

// Descending signed values as ascending unsigned keys.
__global__ void __launch_bounds__(kQ11Block) q11_keys_kernel(const uint32_t* __restrict__ idx,
                                                             const unsigned long long* __restrict__ sums,
                                                             const unsigned long long* n_dev, int64_t limit,
                                                             unsigned long long* __restrict__ keys) {
  const int64_t n = q11_count(n_dev, limit);
  for (int64_t i = (int64_t)blockIdx.x * kQ11Block + threadIdx.x; i < n; i += (int64_t)gridDim.x * kQ11Block)
    keys[i] = ~(sums[idx[i]] ^ (1ull << 63));
}

__global__ void __launch_bounds__(kQ11Block) q11_rows_kernel(const uint32_t* __restrict__ idx,
                                                             const unsigned long long* __restrict__ sums,
                                                             const unsigned long long* n_dev, int64_t limit,
                                                             int32_t min_partkey, bo_tpch_q11_row* __restrict__ rows) {
  const int64_t n = q11_count(n_dev, limit);
  for (int64_t i = (int64_t)blockIdx.x * kQ11Block + threadIdx.x; i < n; i += (int64_t)gridDim.x * kQ11Block) {
    bo_tpch_q11_row r;
    r.ps_partkey = (int32_t)((int64_t)min_partkey + idx[i]);
    r.pad = 0;
    r.value_raw = (int64_t)sums[idx[i]];
    rows[i] = r;
  }
}

int q11_grid(bo_ctx* ctx, int64_t items) {
  const int64_t need = (items + kQ11Block - 1) / kQ11Block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)ctx->num_sms * 8));
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q11_rows(bo_ctx* ctx, const bo_tpch_q11_tables* t, const uint8_t* supp_in_nation_host,
                                int64_t n_supp, double fraction, bo_tpch_q11_row* rows_out, int64_t max_rows,
                                int64_t* n_rows) {
  BO_CHECK_CTX(ctx);
  if (!t || !n_rows || (n_supp > 0 && !supp_in_nation_host) || max_rows < 0 || (max_rows > 0 && !rows_out))
    return set_error(ctx, BO_ERR_INVALID, "q11: null argument");
  if (t->n_partsupp < 0 || n_supp < 0) return set_error(ctx, BO_ERR_INVALID, "q11: negative size");
  *n_rows = 0;
  if (t->n_partsupp == 0 || n_supp == 0) return BO_OK;
  if (t->max_partkey < t->min_partkey) return set_error(ctx, BO_ERR_INVALID, "q11: empty partkey range");
  if (!t->ps_partkey || !t->ps_suppkey || !t->ps_value) return set_error(ctx, BO_ERR_INVALID, "q11: null column");
  const int64_t range = (int64_t)t->max_partkey - t->min_partkey + 1;
  const int64_t tiles = (range + kCompactTile - 1) / kCompactTile;
  size_t total_bytes = 0;
  auto add = [&](size_t b) { total_bytes += (b + 255) & ~size_t(255); };
  add(256);                        // total, then the compacted count
  add(8 * (size_t)range);          // sums
  add((size_t)n_supp);
  add(4 * (size_t)tiles);
  add(4 * (size_t)range);          // compacted indexes
  add(8 * (size_t)range);          // keys
  add(8 * (size_t)range);          // sort scratch
  add(4 * (size_t)range);
  add(sizeof(bo_tpch_q11_row) * (size_t)range);
  void* base = nullptr;
  int rc = region(ctx, "q11_rows_ws", total_bytes, &base);
  if (rc) return rc;
  char* p = static_cast<char*>(base);
  unsigned long long* total = carve<unsigned long long>(p, 32);
  unsigned long long* sums = carve<unsigned long long>(p, (size_t)range);
  uint8_t* in_nation = carve<uint8_t>(p, (size_t)n_supp);
  uint32_t* tile_counts = carve<uint32_t>(p, (size_t)tiles);
  uint32_t* idx = carve<uint32_t>(p, (size_t)range);
  unsigned long long* keys = carve<unsigned long long>(p, (size_t)range);
  unsigned long long* tkeys = carve<unsigned long long>(p, (size_t)range);
  uint32_t* tvals = carve<uint32_t>(p, (size_t)range);
  bo_tpch_q11_row* rows = carve<bo_tpch_q11_row>(p, (size_t)range);
  void* h = nullptr;
  if ((rc = host_stage(ctx, (size_t)n_supp, &h))) return rc;
  std::memcpy(h, supp_in_nation_host, (size_t)n_supp);
  BO_CUDA(ctx, cudaMemcpyAsync(in_nation, h, (size_t)n_supp, cudaMemcpyHostToDevice, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(base, 0, 256 + 8 * (size_t)range, ctx->stream));
  q11_kernel<<<q11_grid(ctx, t->n_partsupp), kQ11Block, 0, ctx->stream>>>(*t, in_nation, n_supp, sums, total,
                                                                           ctx->d_err);
  if ((rc = after_launch(ctx, "q11_kernel"))) return rc;
  unsigned long long* n_out = total + 1;
  if ((rc = ordered_compact(ctx, Q11Kept{sums, total, fraction}, range, tile_counts, idx, n_out))) return rc;
  // Sort and rows read the count on the device; rows into mapped rows_out
  // directly: one synchronisation (a count beyond one cluster sort is sorted
  // again after the read-back).  The overflow word follows the count.
  uint32_t* overflow = reinterpret_cast<uint32_t*>(n_out + 1);
  q11_keys_kernel<<<q11_grid(ctx, range), kQ11Block, 0, ctx->stream>>>(idx, sums, n_out, range, keys);
  if ((rc = after_launch(ctx, "q11_keys_kernel"))) return rc;
  if ((rc = cluster_sort_pairs_counted(ctx, keys, idx, n_out, range, 0, 64, overflow))) return rc;
  bo_tpch_q11_row* direct = max_rows > 0 ? static_cast<bo_tpch_q11_row*>(mapped_device_ptr(rows_out)) : nullptr;
  const int64_t lim = direct ? std::min<int64_t>(max_rows, range) : range;
  auto emit_rows = [&]() {
    q11_rows_kernel<<<q11_grid(ctx, lim), kQ11Block, 0, ctx->stream>>>(idx, sums, n_out, lim, t->min_partkey,
                                                                        direct ? direct : rows);
    return after_launch(ctx, "q11_rows_kernel");
  };
  if ((rc = emit_rows())) return rc;
  int64_t ns = 0;
  bool over = false;
  if ((rc = read_counted(ctx, "q11", n_out, range, &ns, &over))) return rc;
  if (over) {
    if ((rc = radix_sort_pairs(ctx, keys, idx, tkeys, tvals, ns, 0, 64, nullptr))) return rc;
    if ((rc = emit_rows())) return rc;
  }
  const int64_t m = std::min<int64_t>(ns, max_rows);
  if (!direct && m > 0)
    BO_CUDA(ctx, cudaMemcpyAsync(rows_out, rows, sizeof(bo_tpch_q11_row) * (size_t)m, cudaMemcpyDeviceToHost,
                                 ctx->stream));
  if (over || (!direct && m > 0)) {
    uint32_t bits = 0;
    if ((rc = consume_device_errors(ctx, &bits))) return rc;
    if ((rc = device_error_status(ctx, bits, "q11"))) return rc;
  }
  *n_rows = ns;
  return BO_OK;
}

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
