// TPC-H Q10 and Q18 over the storage-plan layout, and the per-order lineitem
// ranges Q10 reads.
//
// Q10 (run_q10, bespoke_tpch/query_q10.cpp:375-585).  The reference walks the
// orders of a three-month date range, sums each one's 'R'-flagged lineitems
// through its range, keeps orders with a non-zero sum, radix-sorts them by
// custkey to total each customer, drops customers without a row or a known
// nation, and radix-sorts by (revenue desc, custkey asc).  Here:
//   orders   one thread per orders row of the range: its lineitem range in a
//            short loop, then one 64-bit atomic into the customer's total and
//            a bit in a customer bitmap (the order's "non-zero" test is kept
//            per order, as in the reference, so totals that cancel to zero
//            still make a group);
//   emit     customers with their bit set, a row and a nation, in ascending
//            custkey order (order-preserving compaction, compact.cuh) -- the
//            order the reference's first sort, by custkey, produces;
//   sort     one stable radix sort by the complemented revenue (64 bits), the
//            reference's own key order (one cluster launch up to 128K rows).
//
// Q18 (run_q18, bespoke_tpch/query_q18.cpp:183-455).
//   sum      sum_qty[orderkey] += l_quantity: each thread takes eight
//            consecutive lineitems (two 16-byte key loads, one 16-byte
//            quantity load) and adds each run of equal keys with one atomic,
//            so lineitems sorted by orderkey cost about one atomic per order;
//   qualify  the reference's dense path reads orderkey k from orders row
//            k - 1 (its dense test looks only at the first and last
//            date-sorted orderkey, :204-206); the other path scans orders
//            rows; both emit (orderkey, orders row) pairs;
//   sort     stable by orderkey, then by (totalprice desc, orderdate asc):
//            the reference's comparator (:438-449).
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "compact.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kTpBlock = 256;
constexpr int kQ18RowsPerThread = 8;

int grid_for(bo_ctx* ctx, int64_t items) {
  const int64_t need = (items + kTpBlock - 1) / kTpBlock;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)ctx->num_sms * 8));
}

// Block-level compaction step: every thread of the block calls it with its
// keep flag; the block reserves its total once.  Returns the output position
// of a kept element.
__device__ __forceinline__ unsigned long long block_reserve(bool keep, unsigned long long* n_out,
                                                            uint32_t* warp_off, unsigned long long* base) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t m = __ballot_sync(0xffffffffu, keep);
  if (lane == 0) warp_off[warp] = __popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kTpBlock / 32; ++w) {
      const uint32_t c = warp_off[w];
      warp_off[w] = t;
      t += c;
    }
    *base = t ? atomicAdd(n_out, (unsigned long long)t) : 0ull;
  }
  __syncthreads();
  const unsigned long long pos = *base + warp_off[warp] + __popc(m & ((1u << lane) - 1u));
  __syncthreads();  // warp_off / base are rewritten by the next call
  return pos;
}

// ------------------------------------------------------------ order ranges --
// Only the first and the last lineitem of each run of equal orderkeys touch
// the range (a neighbour with the same key maps to the same row and lies
// inside the bounds), so sorted lineitems cost two atomics per order.
__global__ void order_range_kernel(const int32_t* __restrict__ l_orderkey, int64_t n,
                                   const int32_t* __restrict__ key_to_row, int64_t n_map, int64_t n_orders,
                                   uint32_t* __restrict__ begin, uint32_t* __restrict__ end) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t key = l_orderkey[i];
    if (key < 0 || (int64_t)key >= n_map) continue;
    const bool first = i == 0 || l_orderkey[i - 1] != key;
    const bool last = i + 1 == n || l_orderkey[i + 1] != key;
    if (!first && !last) continue;
    const int32_t row = key_to_row[key];
    if (row < 0 || (int64_t)row >= n_orders) continue;
    if (first) atomicMin(begin + row, (uint32_t)i);
    if (last) atomicMax(end + row, (uint32_t)(i + 1));
  }
}

// -------------------------------------------------------------------- Q10 --
template <bool kSorted>
__global__ void q10_orders_kernel(const int32_t* __restrict__ o_orderkey, const int32_t* __restrict__ o_custkey,
                                  const int16_t* __restrict__ o_orderdate, const uint32_t* __restrict__ li_begin,
                                  const uint32_t* __restrict__ li_end, int64_t n_orders,
                                  const int32_t* __restrict__ l_orderkey, const uint8_t* __restrict__ l_code,
                                  const int32_t* __restrict__ l_dprice, int64_t n_lineitem, int16_t start,
                                  int16_t end, uint32_t group_lo, uint32_t group_count, int64_t n_map,
                                  const int32_t* __restrict__ key_to_row, const int32_t* __restrict__ c_nationkey,
                                  int64_t n_customer, int32_t nation_bound,
                                  unsigned long long* __restrict__ cust_rev, uint32_t* __restrict__ cust_hit,
                                  uint32_t* err) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_orders;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int16_t d = o_orderdate[i];
    if (d < start || d >= end) continue;
    const int32_t c = o_custkey[i];
    if (c < 0 || (int64_t)c >= n_map) continue;
    const uint32_t e = li_end[i];
    if (e == 0u) continue;
    const uint32_t b = li_begin[i];
    if ((int64_t)e > n_lineitem || b > e) {  // a range that is not one of this lineitem table's
      raise_error(err, kErrValueRange);
      continue;
    }
    const int32_t key = kSorted ? 0 : o_orderkey[i];
    unsigned long long rev = 0;  // int64 sum, wrapping as the reference's
    for (uint32_t j = b; j < e; ++j) {
      if (!kSorted && l_orderkey[j] != key) continue;
      if ((uint32_t)l_code[j] - group_lo >= group_count) continue;
      rev += (unsigned long long)(int64_t)l_dprice[j];
    }
    if (rev == 0ull) continue;
    // Only customers with a row and a known nation give rows (query_q10.cpp:
    // 556-563); their bits are the result's custkeys.
    const int32_t row = __ldg(key_to_row + c);
    if (row < 0 || (int64_t)row >= n_customer) continue;
    const int32_t nk = __ldg(c_nationkey + row);
    if (nk < 0 || nk >= nation_bound) continue;
    atomicAdd(cust_rev + c, rev);
    const uint32_t bit = 1u << (c & 31);
    if (!(__ldg(cust_hit + (c >> 5)) & bit)) atomicOr(cust_hit + (c >> 5), bit);
  }
}

// Revenue descending as an unsigned 64-bit value: the reference's ~revenue key.
__global__ void q10_key2_kernel(const uint32_t* __restrict__ vals, const unsigned long long* __restrict__ cust_rev,
                                const unsigned long long* n_out, unsigned long long* __restrict__ keys) {
  const unsigned long long n = *n_out;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    keys[i] = ~cust_rev[vals[i]];
}

// Per customer row, the host's string offsets and balance (all null: not
// gathered).
struct Q10CustStrings {
  const uint32_t* off[4];  // name, address, phone, comment
  const int32_t* acctbal;
};

__global__ void q10_gather_kernel(const uint32_t* __restrict__ vals, const unsigned long long* __restrict__ cust_rev,
                                  const int32_t* __restrict__ key_to_row, const int32_t* __restrict__ c_nationkey,
                                  Q10CustStrings cs, const unsigned long long* n_out,
                                  bo_tpch_q10_row* __restrict__ out) {
  const unsigned long long n = *n_out;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t c = vals[i];
    const int32_t row = key_to_row[c];
    bo_tpch_q10_row r;
    r.revenue_raw = (int64_t)cust_rev[c];
    r.custkey = (int32_t)c;
    r.cust_row = row;
    r.nationkey = c_nationkey[row];
    r.acctbal_raw = cs.acctbal ? __ldg(cs.acctbal + row) : 0;
    uint32_t b[4] = {0, 0, 0, 0}, l[4] = {0, 0, 0, 0};
    if (cs.off[0]) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        b[k] = __ldg(cs.off[k] + row);
        l[k] = __ldg(cs.off[k] + row + 1) - b[k];
      }
    }
    r.name_begin = b[0];
    r.name_len = l[0];
    r.address_begin = b[1];
    r.address_len = l[1];
    r.phone_begin = b[2];
    r.phone_len = l[2];
    r.comment_begin = b[3];
    r.comment_len = l[3];
    out[i] = r;
  }
}

// The customer strings on the host and the nation names (device table of
// host pointers), for rows the host reads in place.
struct Q10HostStrings {
  const char* data[4];     // name, address, phone, comment bytes (host)
  const uint32_t* off[4];  // their offsets per customer row (device)
  const int32_t* acctbal;
  const bo_host_str* nation_names;
};

// The result rows in their final host form, written straight into mapped
// pinned host memory.  Each thread builds one 96-byte row in shared memory;
// the block then stores its rows as consecutive 16-byte words (one warp
// instruction covers 512 contiguous bytes), so they cross PCIe as full
// writes rather than as many partial ones.  out is 16-byte aligned.
constexpr int kQ10RowsBlock = 128;

__global__ void __launch_bounds__(kQ10RowsBlock) q10_host_rows_kernel(
    const uint32_t* __restrict__ vals, const unsigned long long* __restrict__ cust_rev,
    const int32_t* __restrict__ key_to_row, const int32_t* __restrict__ c_nationkey, Q10HostStrings hs,
    const unsigned long long* n_out, int64_t limit, bo_tpch_q10_host_row* __restrict__ out) {
  __shared__ bo_tpch_q10_host_row stage[kQ10RowsBlock];
  constexpr int kWords = (int)(sizeof(bo_tpch_q10_host_row) / 16);
  static_assert(sizeof(bo_tpch_q10_host_row) % 16 == 0, "rows are whole 16-byte words");
  const unsigned long long nd = *n_out;
  const int64_t n = nd < (unsigned long long)limit ? (int64_t)nd : limit;  // the first min(count, limit) rows
  for (int64_t base = (int64_t)blockIdx.x * kQ10RowsBlock; base < n; base += (int64_t)gridDim.x * kQ10RowsBlock) {
    const int64_t i = base + threadIdx.x;
    if (i < n) {
      const uint32_t c = vals[i];
      const int32_t row = key_to_row[c];
      bo_tpch_q10_host_row r;
      r.custkey = (int32_t)c;
      r.acctbal_raw = __ldg(hs.acctbal + row);
      r.revenue_raw = (int64_t)cust_rev[c];
      bo_host_str* f[4] = {&r.name, &r.address, &r.phone, &r.comment};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint32_t b = __ldg(hs.off[k] + row);
        f[k]->ptr = hs.data[k] + b;
        f[k]->len = __ldg(hs.off[k] + row + 1) - b;
      }
      r.nation_name = hs.nation_names[c_nationkey[row]];
      stage[threadIdx.x] = r;
    }
    __syncthreads();
    const int rows = (int)(n - base < kQ10RowsBlock ? n - base : kQ10RowsBlock);
    const uint4* src = reinterpret_cast<const uint4*>(stage);
    uint4* dst = reinterpret_cast<uint4*>(out + base);
    for (int w = threadIdx.x; w < rows * kWords; w += kQ10RowsBlock) dst[w] = src[w];
    __syncthreads();
  }
}

// -------------------------------------------------------------------- Q18 --
struct Q18Run {
  int32_t key = -1;
  uint32_t sum = 0;  // int32 sum, wrapping as the reference's
};

__device__ __forceinline__ void q18_add(Q18Run& run, int32_t key, int16_t q, int64_t bound, bool dense,
                                        uint32_t* __restrict__ sum, uint32_t* __restrict__ mark, uint32_t* err) {
  if (key < 0 || (int64_t)key >= bound) {  // the reference indexes past its sum array here
    raise_error(err, kErrValueRange);
    return;
  }
  if (dense && q < 0) raise_error(err, kErrValueRange);
  if (key == run.key) {
    run.sum += (uint32_t)(int32_t)q;
    return;
  }
  if (run.key >= 0) {
    atomicAdd(sum + run.key, run.sum);
    if (mark) atomicOr(mark + (run.key >> 5), 1u << (run.key & 31));
  }
  run.key = key;
  run.sum = (uint32_t)(int32_t)q;
}

// mark (dense path with a negative threshold only): orderkeys that occur,
// since the reference qualifies only orderkeys its lineitem scan met.
__global__ void q18_sum_kernel(const int32_t* __restrict__ l_orderkey, const int16_t* __restrict__ l_quantity,
                               int64_t n, int64_t bound, int dense, uint32_t* __restrict__ sum,
                               uint32_t* __restrict__ mark, uint32_t* err) {
  const int64_t groups = n / kQ18RowsPerThread;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t g = tid; g < groups; g += stride) {
    const int4 k0 = __ldg(reinterpret_cast<const int4*>(l_orderkey) + 2 * g);
    const int4 k1 = __ldg(reinterpret_cast<const int4*>(l_orderkey) + 2 * g + 1);
    const int4 qv = __ldg(reinterpret_cast<const int4*>(l_quantity) + g);
    const int32_t keys[kQ18RowsPerThread] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
    const uint32_t qw[4] = {(uint32_t)qv.x, (uint32_t)qv.y, (uint32_t)qv.z, (uint32_t)qv.w};
    Q18Run run;
    for (int j = 0; j < kQ18RowsPerThread; ++j) {
      const int16_t q = (int16_t)(uint16_t)(qw[j >> 1] >> (16 * (j & 1)));
      q18_add(run, keys[j], q, bound, dense != 0, sum, mark, err);
    }
    if (run.key >= 0) {
      atomicAdd(sum + run.key, run.sum);
      if (mark) atomicOr(mark + (run.key >> 5), 1u << (run.key & 31));
    }
  }
  // tail rows, one per thread
  const int64_t i = groups * kQ18RowsPerThread + tid;
  if (i < n) {
    Q18Run run;
    q18_add(run, l_orderkey[i], l_quantity[i], bound, dense != 0, sum, mark, err);
    if (run.key >= 0) {
      atomicAdd(sum + run.key, run.sum);
      if (mark) atomicOr(mark + (run.key >> 5), 1u << (run.key & 31));
    }
  }
}

struct Q18Cust {
  const int32_t* key_to_row;
  int64_t n_map;
  int64_t n_customer;
  bool dense;  // custkey - 1 (dense-orderkey path with dense custkeys)
  __device__ __forceinline__ int32_t row_of(int32_t c) const {
    if (dense) {
      const int64_t r = (int64_t)c - 1;
      return (r >= 0 && r < n_customer) ? (int32_t)r : -1;
    }
    return (c >= 0 && (int64_t)c < n_map) ? key_to_row[c] : -1;
  }
};

// (orderkey, orders row) of every qualifying order.
__global__ void __launch_bounds__(kTpBlock) q18_qualify_kernel(const int32_t* __restrict__ o_orderkey,
                                                               const int32_t* __restrict__ o_custkey,
                                                               int64_t n_orders, int dense, int64_t bound,
                                                               const int32_t* __restrict__ sum,
                                                               const uint32_t* __restrict__ mark,
                                                               int32_t threshold, Q18Cust cust,
                                                               unsigned long long* __restrict__ keys,
                                                               uint32_t* __restrict__ vals,
                                                               unsigned long long* n_out, uint32_t* err) {
  __shared__ uint32_t warp_off[kTpBlock / 32];
  __shared__ unsigned long long base;
  for (int64_t b0 = (int64_t)blockIdx.x * kTpBlock; b0 < n_orders; b0 += (int64_t)gridDim.x * kTpBlock) {
    const int64_t row = b0 + threadIdx.x;
    bool keep = false;
    int32_t key = 0;
    if (row < n_orders) {
      key = dense ? (int32_t)(row + 1) : o_orderkey[row];
      if (key < 0 || (int64_t)key >= bound) {
        raise_error(err, kErrValueRange);
      } else if (sum[key] > threshold && (!mark || ((mark[key >> 5] >> (key & 31)) & 1u))) {
        keep = cust.row_of(o_custkey[row]) >= 0;
      }
    }
    const unsigned long long pos = block_reserve(keep, n_out, warp_off, &base);
    if (keep) {
      keys[pos] = (unsigned long long)((uint32_t)key ^ 0x80000000u);
      vals[pos] = (uint32_t)row;
    }
  }
}

// (totalprice desc, orderdate asc) as one 48-bit ascending key.
__global__ void q18_key2_kernel(const uint32_t* __restrict__ vals, const int32_t* __restrict__ o_totalprice,
                                const int16_t* __restrict__ o_orderdate, const unsigned long long* n_out,
                                unsigned long long* __restrict__ keys) {
  const unsigned long long n = *n_out;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t row = vals[i];
    const uint32_t price_desc = ~((uint32_t)o_totalprice[row] ^ 0x80000000u);
    const uint32_t date_asc = (uint32_t)(uint16_t)o_orderdate[row] ^ 0x8000u;
    keys[i] = ((unsigned long long)price_desc << 16) | date_asc;
  }
}

// The result rows (the first min(*n_out, limit)), built one per thread in
// shared memory and stored as consecutive 16-byte words: out may be mapped
// pinned host memory (whole PCIe writes) or device memory; 16-byte aligned.
constexpr int kQ18RowsBlock = 128;

__global__ void __launch_bounds__(kQ18RowsBlock) q18_gather_kernel(
    const uint32_t* __restrict__ vals, const int32_t* __restrict__ o_orderkey, const int32_t* __restrict__ o_custkey,
    const int16_t* __restrict__ o_orderdate, const int32_t* __restrict__ o_totalprice, int dense,
    const int32_t* __restrict__ sum, Q18Cust cust, const unsigned long long* n_out, unsigned long long limit,
    bo_tpch_q18_row* __restrict__ out) {
  __shared__ bo_tpch_q18_row stage[kQ18RowsBlock];
  constexpr int kWords = (int)(sizeof(bo_tpch_q18_row) / 16);
  static_assert(sizeof(bo_tpch_q18_row) % 16 == 0, "rows are whole 16-byte words");
  const unsigned long long n = *n_out < limit ? *n_out : limit;  // the first min(count, limit) rows
  for (unsigned long long base = (unsigned long long)blockIdx.x * kQ18RowsBlock; base < n;
       base += (unsigned long long)gridDim.x * kQ18RowsBlock) {
    const unsigned long long i = base + threadIdx.x;
    if (i < n) {
      const uint32_t row = vals[i];
      const int32_t key = dense ? (int32_t)(row + 1) : o_orderkey[row];
      const int32_t c = o_custkey[row];
      bo_tpch_q18_row r;
      r.sum_qty_raw = (int64_t)sum[key];
      r.custkey = c;
      r.cust_row = cust.row_of(c);
      r.orderkey = key;
      r.totalprice_raw = o_totalprice[row];
      r.orderdate_offset = o_orderdate[row];
      r.pad0 = 0;
      r.pad1 = 0;
      stage[threadIdx.x] = r;
    }
    __syncthreads();
    const int rows = (int)(n - base < kQ18RowsBlock ? n - base : kQ18RowsBlock);
    const uint4* src = reinterpret_cast<const uint4*>(stage);
    uint4* dst = reinterpret_cast<uint4*>(out + base);
    for (int w = threadIdx.x; w < rows * kWords; w += kQ18RowsBlock) dst[w] = src[w];
    __syncthreads();
  }
}

template <class Row>
int finish_rows(bo_ctx* ctx, const char* op, const unsigned long long* n_out, const Row* rows, Row* out_host,
                int64_t max_rows, int64_t* n_rows) {
  unsigned long long n = 0;
  BO_CUDA(ctx, cudaMemcpyAsync(&n, n_out, 8, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  int rc = consume_device_errors(ctx, &bits);  // synchronises the stream
  if (rc) return rc;
  if ((rc = device_error_status(ctx, bits, op))) return rc;
  *n_rows = (int64_t)n;
  const int64_t m = std::min<int64_t>((int64_t)n, max_rows);
  if (m > 0) {
    BO_CUDA(ctx, cudaMemcpyAsync(out_host, rows, sizeof(Row) * (size_t)m, cudaMemcpyDeviceToHost, ctx->stream));
    BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return BO_OK;
}

// The same with the row count already on the host: the rows are copied
// before the one synchronisation.
template <class Row>
int finish_known_rows(bo_ctx* ctx, const char* op, int64_t n, const Row* rows, Row* out_host, int64_t max_rows,
                      int64_t* n_rows) {
  const int64_t m = std::min<int64_t>(n, max_rows);
  if (m > 0)
    BO_CUDA(ctx, cudaMemcpyAsync(out_host, rows, sizeof(Row) * (size_t)m, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  int rc = consume_device_errors(ctx, &bits);  // synchronises the stream
  if (rc) return rc;
  if ((rc = device_error_status(ctx, bits, op))) return rc;
  *n_rows = n;
  return BO_OK;
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_order_ranges(bo_ctx* ctx, const int32_t* l_orderkey, int64_t n_lineitem,
                                    const int32_t* orderkey_to_row, int64_t n_orderkey_map, int64_t n_orders,
                                    uint32_t* begin, uint32_t* end) {
  BO_CHECK_CTX(ctx);
  if (n_lineitem < 0 || n_orderkey_map < 0 || n_orders < 0)
    return set_error(ctx, BO_ERR_INVALID, "order_ranges: negative size");
  if (n_lineitem >= 0xffffffffll) return set_error(ctx, BO_ERR_INVALID, "order_ranges: 2^32 or more lineitems");
  if ((n_lineitem > 0 && !l_orderkey) || (n_orderkey_map > 0 && !orderkey_to_row) ||
      (n_orders > 0 && (!begin || !end)))
    return set_error(ctx, BO_ERR_INVALID, "order_ranges: null argument");
  if (n_orders == 0) return BO_OK;
  BO_CUDA(ctx, cudaMemsetAsync(begin, 0xff, 4 * (size_t)n_orders, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(end, 0, 4 * (size_t)n_orders, ctx->stream));
  if (n_lineitem == 0 || n_orderkey_map == 0) return BO_OK;
  order_range_kernel<<<grid_for(ctx, n_lineitem), kTpBlock, 0, ctx->stream>>>(l_orderkey, n_lineitem,
                                                                              orderkey_to_row, n_orderkey_map,
                                                                              n_orders, begin, end);
  return after_launch(ctx, "order_range_kernel");
}

namespace {
// Q10 up to its sorted result: r->vals holds the result custkeys in row order,
// r->rev the revenue per custkey, r->n the row count (0: no rows; then the
// other fields are unset).
// counted: the sort reads the count on the device (one cluster launch); n is
// then -1 and a count beyond the cluster sets *overflow (see q10_resort).
struct Q10Sorted {
  uint32_t* vals;
  const unsigned long long* rev;
  const unsigned long long* n_out;
  bo_tpch_q10_row* rows;  // workspace for the rows of bo_tpch_q10
  int64_t n;
  unsigned long long *keys, *tkeys;
  uint32_t* tvals;
  uint32_t* overflow;
};

int q10_run(bo_ctx* ctx, const bo_tpch_q10_tables* t, int16_t start_offset, int16_t end_offset, int32_t group_lo,
            int32_t group_count, bool counted, Q10Sorted* r) {
  *r = Q10Sorted{};
  if (t->n_orders < 0 || t->n_lineitem < 0 || t->n_custkey_map < 0 || t->n_customer < 0 || t->nation_bound < 0 ||
      group_count < 0)
    return set_error(ctx, BO_ERR_INVALID, "q10: negative size");
  if (t->n_custkey_map > 0x80000000ll) return set_error(ctx, BO_ERR_INVALID, "q10: custkey map beyond int32 keys");
  if ((t->n_orders > 0 && (!t->o_orderkey || !t->o_custkey || !t->o_orderdate || !t->o_li_begin || !t->o_li_end)) ||
      (t->n_lineitem > 0 && (!t->l_orderkey || !t->l_returnflag_linestatus || !t->l_discounted_price)) ||
      (t->n_custkey_map > 0 && !t->custkey_to_row) || (t->n_customer > 0 && !t->c_nationkey))
    return set_error(ctx, BO_ERR_INVALID, "q10: null column");
  {
    const bool any = t->c_name_offsets || t->c_address_offsets || t->c_phone_offsets || t->c_comment_offsets;
    const bool all = t->c_name_offsets && t->c_address_offsets && t->c_phone_offsets && t->c_comment_offsets;
    if (any && !all) return set_error(ctx, BO_ERR_INVALID, "q10: give all four string offset columns or none");
  }
  const int64_t nm = t->n_custkey_map;
  if (group_lo < 0 || t->n_orders == 0 || nm == 0 || t->n_lineitem == 0) return BO_OK;
  const int64_t hit_words = (nm + 31) / 32;
  size_t total = 0;
  auto add = [&](size_t b) { total += (b + 255) & ~size_t(255); };
  add(8 * (size_t)nm);  // revenue per custkey
  add(4 * (size_t)hit_words);
  add(8 * (size_t)nm);  // keys
  add(4 * (size_t)nm);  // vals
  add(8 * (size_t)nm);  // tmp keys
  add(4 * (size_t)nm);  // tmp vals
  add(sizeof(bo_tpch_q10_row) * (size_t)nm);
  const int64_t tiles = (hit_words + kBitmapTileWords - 1) / kBitmapTileWords;
  add(4 * (size_t)std::max<int64_t>(tiles, 1));  // bitmap compaction's tile counts
  add(64);
  void* basep = nullptr;
  int rc = region(ctx, "q10_ws", total, &basep);
  if (rc) return rc;
  char* p = static_cast<char*>(basep);
  auto* rev = carve<unsigned long long>(p, (size_t)nm);
  auto* hit = carve<uint32_t>(p, (size_t)hit_words);
  auto* keys = carve<unsigned long long>(p, (size_t)nm);
  auto* vals = carve<uint32_t>(p, (size_t)nm);
  auto* tkeys = carve<unsigned long long>(p, (size_t)nm);
  auto* tvals = carve<uint32_t>(p, (size_t)nm);
  auto* rows = carve<bo_tpch_q10_row>(p, (size_t)nm);
  auto* tile_counts = carve<uint32_t>(p, (size_t)std::max<int64_t>(tiles, 1));
  auto* n_out = carve<unsigned long long>(p, 8);
  BO_CUDA(ctx, cudaMemsetAsync(rev, 0, 8 * (size_t)nm, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(hit, 0, 4 * (size_t)hit_words, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(n_out, 0, 16, ctx->stream));  // the count and the sort's overflow word
  const int og = grid_for(ctx, t->n_orders);
  if (t->lineitem_orderkey_sorted)
    q10_orders_kernel<true><<<og, kTpBlock, 0, ctx->stream>>>(
        t->o_orderkey, t->o_custkey, t->o_orderdate, t->o_li_begin, t->o_li_end, t->n_orders, t->l_orderkey,
        t->l_returnflag_linestatus, t->l_discounted_price, t->n_lineitem, start_offset, end_offset,
        (uint32_t)group_lo, (uint32_t)group_count, nm, t->custkey_to_row, t->c_nationkey, t->n_customer,
        t->nation_bound, rev, hit, ctx->d_err);
  else
    q10_orders_kernel<false><<<og, kTpBlock, 0, ctx->stream>>>(
        t->o_orderkey, t->o_custkey, t->o_orderdate, t->o_li_begin, t->o_li_end, t->n_orders, t->l_orderkey,
        t->l_returnflag_linestatus, t->l_discounted_price, t->n_lineitem, start_offset, end_offset,
        (uint32_t)group_lo, (uint32_t)group_count, nm, t->custkey_to_row, t->c_nationkey, t->n_customer,
        t->nation_bound, rev, hit, ctx->d_err);
  if ((rc = after_launch(ctx, "q10_orders_kernel"))) return rc;
  // Customers with revenue in the window, in ascending custkey order (the set
  // bits of the hit bitmap): the order the reference's first LSD sort by
  // custkey gives (query_q10.cpp:318-345), so only the revenue sort remains.
  if ((rc = bitmap_compact(ctx, hit, hit_words, tile_counts, vals, n_out))) return rc;
  // The result's size, read back once: up to 128K rows sort in one cluster
  // launch instead of a pass sequence sized for every customer.
  uint32_t* overflow = reinterpret_cast<uint32_t*>(n_out + 1);
  if (counted) {
    q10_key2_kernel<<<grid_for(ctx, nm), kTpBlock, 0, ctx->stream>>>(vals, rev, n_out, keys);
    if ((rc = after_launch(ctx, "q10_key2_kernel"))) return rc;
    if ((rc = cluster_sort_pairs_counted(ctx, keys, vals, n_out, nm, 0, 64, overflow))) return rc;
    *r = Q10Sorted{vals, rev, n_out, rows, -1, keys, tkeys, tvals, overflow};
    return BO_OK;
  }
  int64_t ns = 0;
  if ((rc = read_device_count(ctx, n_out, nm, &ns))) return rc;
  q10_key2_kernel<<<grid_for(ctx, std::max<int64_t>(ns, 1)), kTpBlock, 0, ctx->stream>>>(vals, rev, n_out, keys);
  if ((rc = after_launch(ctx, "q10_key2_kernel"))) return rc;
  if ((rc = radix_sort_pairs(ctx, keys, vals, tkeys, tvals, ns, 0, 64, nullptr))) return rc;
  *r = Q10Sorted{vals, rev, n_out, rows, ns, keys, tkeys, tvals, overflow};
  return BO_OK;
}
}  // namespace

extern "C" int bo_tpch_q10(bo_ctx* ctx, const bo_tpch_q10_tables* t, int16_t start_offset, int16_t end_offset,
                           int32_t group_lo, int32_t group_count, bo_tpch_q10_row* out_host, int64_t max_rows,
                           int64_t* n_rows) {
  BO_CHECK_CTX(ctx);
  if (!t || !n_rows || max_rows < 0 || (max_rows > 0 && !out_host))
    return set_error(ctx, BO_ERR_INVALID, "q10: null argument");
  *n_rows = 0;
  Q10Sorted r{};
  int rc = q10_run(ctx, t, start_offset, end_offset, group_lo, group_count, false, &r);
  if (rc) return rc;
  if (r.n == 0) return finish_known_rows<bo_tpch_q10_row>(ctx, "q10", 0, nullptr, out_host, max_rows, n_rows);
  const Q10CustStrings cs{{t->c_name_offsets, t->c_address_offsets, t->c_phone_offsets, t->c_comment_offsets},
                          t->c_acctbal};
  q10_gather_kernel<<<grid_for(ctx, r.n), kTpBlock, 0, ctx->stream>>>(r.vals, r.rev, t->custkey_to_row,
                                                                      t->c_nationkey, cs, r.n_out, r.rows);
  if ((rc = after_launch(ctx, "q10_gather_kernel"))) return rc;
  return finish_known_rows(ctx, "q10", r.n, r.rows, out_host, max_rows, n_rows);
}

extern "C" int bo_tpch_q10_host_rows(bo_ctx* ctx, const bo_tpch_q10_tables* t, int16_t start_offset,
                                     int16_t end_offset, int32_t group_lo, int32_t group_count,
                                     const bo_tpch_q10_host_strings* hs, bo_tpch_q10_host_row* rows_mapped,
                                     int64_t max_rows, int64_t* n_rows) {
  BO_CHECK_CTX(ctx);
  if (!t || !hs || !n_rows || max_rows < 0 || (max_rows > 0 && !rows_mapped))
    return set_error(ctx, BO_ERR_INVALID, "q10: null argument");
  *n_rows = 0;
  if (!t->c_name_offsets || !t->c_address_offsets || !t->c_phone_offsets || !t->c_comment_offsets || !t->c_acctbal ||
      !hs->name_data || !hs->address_data || !hs->phone_data || !hs->comment_data ||
      (hs->n_nation > 0 && !hs->nation_names))
    return set_error(ctx, BO_ERR_INVALID, "q10: host rows need the string offsets, balances and host strings");
  if (hs->n_nation < 0 || hs->n_nation < t->nation_bound)
    return set_error(ctx, BO_ERR_INVALID, "q10: %d nation names for nation keys below %d", (int)hs->n_nation,
                     (int)t->nation_bound);
  bo_tpch_q10_host_row* dev_rows = nullptr;
  if (max_rows > 0) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, rows_mapped) != cudaSuccess || attr.type != cudaMemoryTypeHost ||
        !attr.devicePointer) {
      cudaGetLastError();
      return set_error(ctx, BO_ERR_INVALID, "q10: rows_mapped is not mapped pinned host memory");
    }
    dev_rows = static_cast<bo_tpch_q10_host_row*>(attr.devicePointer);
    if (!aligned16(dev_rows)) return set_error(ctx, BO_ERR_INVALID, "q10: rows_mapped is not 16-byte aligned");
  }
  Q10Sorted r{};
  int rc = q10_run(ctx, t, start_offset, end_offset, group_lo, group_count, true, &r);
  if (rc) return rc;
  uint32_t bits = 0;
  if (!r.vals) {  // nothing ran: no rows
    if ((rc = consume_device_errors(ctx, &bits))) return rc;
    return device_error_status(ctx, bits, "q10");
  }
  // The nation names, as a small device table.
  const size_t nb = sizeof(bo_host_str) * (size_t)hs->n_nation;
  void* dn = nullptr;
  void* h = nullptr;
  if ((rc = region(ctx, "q10_nation_names", std::max<size_t>(nb, 16), &dn))) return rc;
  if ((rc = host_stage(ctx, std::max<size_t>(nb, 16) + 16, &h))) return rc;
  if (nb) {
    std::memcpy(h, hs->nation_names, nb);
    BO_CUDA(ctx, cudaMemcpyAsync(dn, h, nb, cudaMemcpyHostToDevice, ctx->stream));
  }
  const Q10HostStrings hsd{{hs->name_data, hs->address_data, hs->phone_data, hs->comment_data},
                           {t->c_name_offsets, t->c_address_offsets, t->c_phone_offsets, t->c_comment_offsets},
                           t->c_acctbal, static_cast<const bo_host_str*>(dn)};
  const int64_t lim = std::min<int64_t>(max_rows, t->n_custkey_map);
  auto rows_out = [&]() {
    if (lim <= 0) return (int)BO_OK;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((lim + kQ10RowsBlock - 1) / kQ10RowsBlock,
                                                                  (int64_t)ctx->num_sms * 8));
    q10_host_rows_kernel<<<grid, kQ10RowsBlock, 0, ctx->stream>>>(r.vals, r.rev, t->custkey_to_row, t->c_nationkey,
                                                                   hsd, r.n_out, lim, dev_rows);
    return after_launch(ctx, "q10_host_rows_kernel");
  };
  if ((rc = rows_out())) return rc;
  // One synchronisation: the count and the sort's overflow word come back
  // with the error word.
  char* cnt_h = static_cast<char*>(h) + ((std::max<size_t>(nb, 16) + 15) & ~size_t(15));
  BO_CUDA(ctx, cudaMemcpyAsync(cnt_h, r.n_out, 16, cudaMemcpyDeviceToHost, ctx->stream));
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // synchronises the stream: the rows have landed
  if ((rc = device_error_status(ctx, bits, "q10"))) return rc;
  const int64_t ns = (int64_t)std::min<unsigned long long>(*reinterpret_cast<const unsigned long long*>(cnt_h),
                                                           (unsigned long long)t->n_custkey_map);
  if (*reinterpret_cast<const uint32_t*>(cnt_h + 8) != 0u) {
    // More rows than one cluster sorts: the pass sequence with the count now known, then the rows again.
    if ((rc = radix_sort_pairs(ctx, r.keys, r.vals, r.tkeys, r.tvals, ns, 0, 64, nullptr))) return rc;
    if ((rc = rows_out())) return rc;
    if ((rc = consume_device_errors(ctx, &bits))) return rc;
    if ((rc = device_error_status(ctx, bits, "q10"))) return rc;
  }
  *n_rows = ns;
  return BO_OK;
}

namespace {
// counted: both sorts read the result count on the device and the rows go
// straight into out_host where it is mapped pinned memory (one
// synchronisation); a count beyond one cluster sort reruns the whole query
// with the count read back before the sorts (the second sort's keys replace
// the first's, so the rerun starts over).
int q18_run(bo_ctx* ctx, const bo_tpch_q18_tables* t, int32_t quantity_threshold, bo_tpch_q18_row* out_host,
            int64_t max_rows, int64_t* n_rows, bool counted) {
  if (!t || !n_rows || max_rows < 0 || (max_rows > 0 && !out_host))
    return set_error(ctx, BO_ERR_INVALID, "q18: null argument");
  if (t->n_orders < 0 || t->n_lineitem < 0 || t->n_custkey_map < 0 || t->n_customer < 0 || t->orderkey_bound < 0)
    return set_error(ctx, BO_ERR_INVALID, "q18: negative size");
  if (t->n_orders > 0x7fffffffll || t->orderkey_bound > 0x80000000ll || t->n_custkey_map > 0x80000000ll)
    return set_error(ctx, BO_ERR_INVALID, "q18: sizes beyond int32 keys");
  if ((t->n_orders > 0 && (!t->o_orderkey || !t->o_custkey || !t->o_orderdate || !t->o_totalprice)) ||
      (t->n_lineitem > 0 && (!t->l_orderkey || !t->l_quantity)) || (t->n_custkey_map > 0 && !t->custkey_to_row))
    return set_error(ctx, BO_ERR_INVALID, "q18: null column");
  if ((reinterpret_cast<uintptr_t>(t->l_orderkey) | reinterpret_cast<uintptr_t>(t->l_quantity)) & 15u)
    return set_error(ctx, BO_ERR_INVALID, "q18: lineitem columns must be 16-byte aligned");
  *n_rows = 0;
  const bool dense = t->dense_orderkeys != 0;
  // Empty cases of :207-213, :295-302 and :324-330.
  if (dense && (t->n_orders == 0 || t->n_customer == 0)) return BO_OK;
  if (!dense && t->orderkey_bound == 0) return BO_OK;
  if (t->n_custkey_map == 0 && !(dense && t->dense_custkeys)) return BO_OK;
  const int64_t no = t->n_orders;
  const int64_t bound = dense ? no + 1 : t->orderkey_bound;
  const bool use_mark = dense && quantity_threshold < 0;
  const int64_t mark_words = use_mark ? (bound + 31) / 32 : 0;
  const int64_t cap = std::max<int64_t>(no, 1);
  size_t total = 0;
  auto add = [&](size_t b) { total += (b + 255) & ~size_t(255); };
  add(4 * (size_t)bound);
  add(4 * (size_t)std::max<int64_t>(mark_words, 1));
  add(8 * (size_t)cap);
  add(4 * (size_t)cap);
  add(8 * (size_t)cap);
  add(4 * (size_t)cap);
  add(sizeof(bo_tpch_q18_row) * (size_t)cap);
  add(64);
  void* basep = nullptr;
  int rc = region(ctx, "q18_ws", total, &basep);
  if (rc) return rc;
  char* p = static_cast<char*>(basep);
  auto* sum = carve<int32_t>(p, (size_t)bound);
  auto* mark = carve<uint32_t>(p, (size_t)std::max<int64_t>(mark_words, 1));
  auto* keys = carve<unsigned long long>(p, (size_t)cap);
  auto* vals = carve<uint32_t>(p, (size_t)cap);
  auto* tkeys = carve<unsigned long long>(p, (size_t)cap);
  auto* tvals = carve<uint32_t>(p, (size_t)cap);
  auto* rows = carve<bo_tpch_q18_row>(p, (size_t)cap);
  auto* n_out = carve<unsigned long long>(p, 8);
  BO_CUDA(ctx, cudaMemsetAsync(sum, 0, 4 * (size_t)bound, ctx->stream));
  if (use_mark) BO_CUDA(ctx, cudaMemsetAsync(mark, 0, 4 * (size_t)mark_words, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(n_out, 0, 16, ctx->stream));  // the count and the sorts' overflow word
  if (t->n_lineitem > 0) {
    const int64_t threads = t->n_lineitem / kQ18RowsPerThread + kQ18RowsPerThread;
    q18_sum_kernel<<<grid_for(ctx, threads), kTpBlock, 0, ctx->stream>>>(
        t->l_orderkey, t->l_quantity, t->n_lineitem, bound, dense ? 1 : 0, reinterpret_cast<uint32_t*>(sum),
        use_mark ? mark : nullptr, ctx->d_err);
    if ((rc = after_launch(ctx, "q18_sum_kernel"))) return rc;
  }
  if (no == 0) return finish_rows(ctx, "q18", n_out, rows, out_host, max_rows, n_rows);
  const Q18Cust cust{t->custkey_to_row, t->n_custkey_map, t->n_customer, dense && t->dense_custkeys != 0};
  q18_qualify_kernel<<<grid_for(ctx, no), kTpBlock, 0, ctx->stream>>>(
      t->o_orderkey, t->o_custkey, no, dense ? 1 : 0, bound, sum, use_mark ? mark : nullptr, quantity_threshold,
      cust, keys, vals, n_out, ctx->d_err);
  if ((rc = after_launch(ctx, "q18_qualify_kernel"))) return rc;
  uint32_t* overflow = reinterpret_cast<uint32_t*>(n_out + 1);
  int64_t ns = 0;
  if (!counted) {  // the result's size, read back once before the sorts
    if ((rc = read_device_count(ctx, n_out, cap, &ns))) return rc;
    if ((rc = radix_sort_pairs(ctx, keys, vals, tkeys, tvals, ns, 0, 32, nullptr))) return rc;
  } else if ((rc = cluster_sort_pairs_counted(ctx, keys, vals, n_out, cap, 0, 32, overflow))) {
    return rc;
  }
  q18_key2_kernel<<<grid_for(ctx, no), kTpBlock, 0, ctx->stream>>>(vals, t->o_totalprice, t->o_orderdate, n_out,
                                                                     keys);
  if ((rc = after_launch(ctx, "q18_key2_kernel"))) return rc;
  if (!counted) {
    if ((rc = radix_sort_pairs(ctx, keys, vals, tkeys, tvals, ns, 0, 48, nullptr))) return rc;
  } else if ((rc = cluster_sort_pairs_counted(ctx, keys, vals, n_out, cap, 0, 48, overflow))) {
    return rc;
  }
  bo_tpch_q18_row* direct =
      (counted && max_rows > 0) ? static_cast<bo_tpch_q18_row*>(mapped_device_ptr(out_host)) : nullptr;
  const int64_t lim = direct ? std::min<int64_t>(max_rows, cap) : cap;
  const int ggrid = (int)std::max<int64_t>(1, std::min<int64_t>((lim + kQ18RowsBlock - 1) / kQ18RowsBlock,
                                                                  (int64_t)ctx->num_sms * 8));
  q18_gather_kernel<<<ggrid, kQ18RowsBlock, 0, ctx->stream>>>(vals, t->o_orderkey, t->o_custkey, t->o_orderdate,
                                                              t->o_totalprice, dense ? 1 : 0, sum, cust, n_out,
                                                              (unsigned long long)lim, direct ? direct : rows);
  if ((rc = after_launch(ctx, "q18_gather_kernel"))) return rc;
  if (!counted) return finish_known_rows(ctx, "q18", ns, rows, out_host, max_rows, n_rows);
  bool over = false;
  if ((rc = read_counted(ctx, "q18", n_out, cap, &ns, &over))) return rc;
  if (over) return q18_run(ctx, t, quantity_threshold, out_host, max_rows, n_rows, false);
  if (direct) {
    *n_rows = ns;
    return BO_OK;
  }
  return finish_known_rows(ctx, "q18", ns, rows, out_host, max_rows, n_rows);
}
}  // namespace

extern "C" int bo_tpch_q18(bo_ctx* ctx, const bo_tpch_q18_tables* t, int32_t quantity_threshold,
                           bo_tpch_q18_row* out_host, int64_t max_rows, int64_t* n_rows) {
  BO_CHECK_CTX(ctx);
  return q18_run(ctx, t, quantity_threshold, out_host, max_rows, n_rows, true);
}
