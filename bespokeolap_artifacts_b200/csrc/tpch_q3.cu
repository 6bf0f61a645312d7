// TPC-H Q3 over the storage-plan layout: run_q3 of bespoke_tpch/query_q3.cpp:153-365.
//
// The reference walks the orders sorted by date, takes the qualifying ones
// (orderdate < D, customer in the segment; :207-322) and sums each one's
// lineitems with shipdate > D through its CSR range (:219-260), then sorts all
// resulting orders by revenue desc, orderdate asc (:348-355).  On the GPU the
// same result comes from four data-parallel passes and a sort:
//   cust   segment membership as a bitmap over custkey (:182-204);
//   orders one 32-row bitmap word per warp iteration: orderdate < D and the
//          customer's bit (:311-322); no atomics;
//   lines  every lineitem with shipdate > D finds its order row through
//          orderkey_to_row (the map the reference's CSR ranges are built from,
//          bespoke_tpch/builder_impl.cpp:930-990) and, if that order
//          qualifies, adds its discounted price and a count with 64-bit
//          atomics (only the ~2% of lineitems that pass both filters do);
//   compact orders with at least one such lineitem (`has_lineitem`, :248):
//          the lineitem pass sets the orderkey's bit when it counts an
//          order's first lineitem, and the set bits come out in ascending
//          orderkey order (bitmap compaction, compact.cuh);
//   sort   one stable radix sort by (revenue desc, orderdate asc) -- one
//          cluster launch that reads the result's size on the device, up to
//          128K result rows (more: the pass sequence, sized after a read-back);
//   rows   staged in shared memory and stored straight into the caller's
//          mapped pinned memory where it is that, so the query synchronises
//          once.  The reference's std::sort
//          leaves rows equal in both keys in unspecified order; here they keep
//          orderkey order, a canonical form of the same result.
#include <algorithm>

#include "common.cuh"
#include "compact.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ3Block = 256;
constexpr unsigned long long kRevBits = 47;  // revenue < 2^47 (checked) so (rev, date) packs into 63 bits

__global__ void q3_cust_kernel(const int32_t* __restrict__ custkey, const uint16_t* __restrict__ seg, int64_t n,
                               int32_t segment_code, int32_t bound, uint32_t* __restrict__ mask) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if ((int32_t)seg[i] != segment_code) continue;
    const int32_t k = custkey[i];
    if (k >= 0 && k < bound) atomicOr(mask + (k >> 5), 1u << (k & 31));
  }
}

// Warp w of the grid owns order rows [32w, 32w + 32): one qualification word.
__global__ void q3_orders_kernel(const int32_t* __restrict__ o_custkey, const int16_t* __restrict__ o_orderdate,
                                 int64_t n, int16_t date_offset, int32_t bound, const uint32_t* __restrict__ mask,
                                 uint32_t* __restrict__ qual) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w * 32 < n; w += warps) {
    const int64_t i = w * 32 + lane;
    bool q = false;
    if (i < n && o_orderdate[i] < date_offset) {
      const int32_t c = o_custkey[i];
      q = c >= 0 && c < bound && ((mask[c >> 5] >> (c & 31)) & 1u);
    }
    const uint32_t word = __ballot_sync(0xffffffffu, q);
    if (lane == 0) qual[w] = word;
  }
}

__global__ void q3_lineitem_kernel(const int32_t* __restrict__ l_orderkey, const int16_t* __restrict__ l_shipdate,
                                   const int32_t* __restrict__ l_dprice, int64_t n, int16_t date_offset,
                                   const int32_t* __restrict__ key_to_row, int64_t n_map, int64_t n_orders,
                                   const uint32_t* __restrict__ qual, unsigned long long* __restrict__ rev,
                                   uint32_t* __restrict__ cnt, uint32_t* __restrict__ kept) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (l_shipdate[i] <= date_offset) continue;
    const int32_t key = l_orderkey[i];
    if (key < 0 || (int64_t)key >= n_map) continue;
    const int32_t row = key_to_row[key];
    if (row < 0 || (int64_t)row >= n_orders) continue;
    if (!((qual[row >> 5] >> (row & 31)) & 1u)) continue;
    atomicAdd(rev + row, (unsigned long long)(int64_t)l_dprice[i]);
    if (atomicAdd(cnt + row, 1u) == 0u) atomicOr(kept + (key >> 5), 1u << (key & 31));
  }
}

// Orders with a counted lineitem -> (orderkey, row) pairs; one reservation per block.
// vals[i] holds a kept orderkey on entry and its order row on return.
__global__ void q3_key2_kernel(uint32_t* __restrict__ vals, const int32_t* __restrict__ key_to_row,
                               const unsigned long long* __restrict__ rev, const int16_t* __restrict__ o_orderdate,
                               const unsigned long long* n_out, unsigned long long* __restrict__ keys, uint32_t* err) {
  const unsigned long long n = *n_out;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t row = (uint32_t)__ldg(key_to_row + vals[i]);  // valid: the lineitem pass marked it
    vals[i] = row;
    const unsigned long long r = rev[row];
    if (r >> kRevBits) raise_error(err, kErrValueRange);
    const unsigned long long inv = ((1ull << kRevBits) - 1ull) - (r & ((1ull << kRevBits) - 1ull));
    keys[i] = (inv << 16) | (unsigned long long)(uint16_t)(o_orderdate[row] + 32768);
  }
}

// The result rows (the first min(*n_out, limit)), one per thread, staged in
// shared memory and stored as consecutive 16-byte words: out may be mapped
// pinned host memory (the rows then cross PCIe as whole writes) or device
// memory.  out is 16-byte aligned.
constexpr int kQ3RowsBlock = 128;

__global__ void __launch_bounds__(kQ3RowsBlock) q3_gather_kernel(
    const uint32_t* __restrict__ vals, const unsigned long long* __restrict__ rev,
    const int32_t* __restrict__ o_orderkey, const int16_t* __restrict__ o_orderdate,
    const int32_t* __restrict__ o_shippriority, const unsigned long long* n_out, int64_t limit,
    bo_tpch_q3_row* __restrict__ out) {
  __shared__ bo_tpch_q3_row stage[kQ3RowsBlock];
  static_assert((sizeof(bo_tpch_q3_row) * kQ3RowsBlock) % 16 == 0, "a block's rows are whole 16-byte words");
  const unsigned long long nd = *n_out;
  const int64_t n = nd < (unsigned long long)limit ? (int64_t)nd : limit;
  for (int64_t base = (int64_t)blockIdx.x * kQ3RowsBlock; base < n; base += (int64_t)gridDim.x * kQ3RowsBlock) {
    const int64_t i = base + threadIdx.x;
    if (i < n) {
      const uint32_t row = vals[i];
      bo_tpch_q3_row r;
      r.revenue_raw = (int64_t)rev[row];
      r.orderkey = o_orderkey[row];
      r.shippriority = o_shippriority ? o_shippriority[row] : 0;
      r.orderdate_offset = o_orderdate[row];
      r.pad0 = 0;
      r.pad1 = 0;
      stage[threadIdx.x] = r;
    }
    __syncthreads();
    const int rows = (int)(n - base < kQ3RowsBlock ? n - base : kQ3RowsBlock);
    const int words = (int)((sizeof(bo_tpch_q3_row) * rows + 15) / 16);  // the tail word may carry pad bytes
    const uint4* src = reinterpret_cast<const uint4*>(stage);
    uint4* dst = reinterpret_cast<uint4*>(out + base);
    if (rows == kQ3RowsBlock || (sizeof(bo_tpch_q3_row) * rows) % 16 == 0) {
      for (int w = threadIdx.x; w < words; w += kQ3RowsBlock) dst[w] = src[w];
    } else {  // a ragged last block: 8-byte words, so nothing past row n - 1 is written
      const uint2* s2 = reinterpret_cast<const uint2*>(stage);
      uint2* d2 = reinterpret_cast<uint2*>(out + base);
      for (int w = threadIdx.x; w < (int)(sizeof(bo_tpch_q3_row) / 8) * rows; w += kQ3RowsBlock) d2[w] = s2[w];
    }
    __syncthreads();
  }
}

// The lineitem pass, 8 rows per thread per step: one 16-byte load of 8
// shipdates, and for a step with any row past the date one 32-byte pair of
// orderkey loads; the map lookups of the passing rows are all issued before
// any is used (independent loads in flight), then the qualification bits,
// then the atomics.  Columns 16-byte aligned (checked by the caller); the
// last n % 8 rows go through the scalar loop.
__global__ void __launch_bounds__(kQ3Block) q3_lineitem_v8_kernel(
    const int32_t* __restrict__ l_orderkey, const int16_t* __restrict__ l_shipdate,
    const int32_t* __restrict__ l_dprice, int64_t n, int16_t date_offset, const int32_t* __restrict__ key_to_row,
    int64_t n_map, int64_t n_orders, const uint32_t* __restrict__ qual, unsigned long long* __restrict__ rev,
    uint32_t* __restrict__ cnt, uint32_t* __restrict__ kept) {
  const int64_t chunks = n >> 3;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t c = tid; c < chunks; c += stride) {
    const int64_t r0 = c << 3;
    const int4 sd = ld_stream_v4(l_shipdate + r0);
    const uint32_t sw[4] = {(uint32_t)sd.x, (uint32_t)sd.y, (uint32_t)sd.z, (uint32_t)sd.w};
    uint32_t pass = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int16_t d = (int16_t)((sw[k >> 1] >> (16 * (k & 1))) & 0xffffu);
      pass |= (uint32_t)(d > date_offset) << k;
    }
    if (!pass) continue;
    const int4 k0 = ld_stream_v4(l_orderkey + r0), k1 = ld_stream_v4(l_orderkey + r0 + 4);
    const int32_t key[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
    int32_t row[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      row[k] = -1;
      if (((pass >> k) & 1u) && key[k] >= 0 && (int64_t)key[k] < n_map) row[k] = __ldg(key_to_row + key[k]);
    }
    uint32_t word[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const bool in = row[k] >= 0 && (int64_t)row[k] < n_orders;
      word[k] = in ? __ldg(qual + (row[k] >> 5)) : 0u;
      if (!in) row[k] = -1;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (row[k] < 0 || !((word[k] >> (row[k] & 31)) & 1u)) continue;
      atomicAdd(rev + row[k], (unsigned long long)(int64_t)__ldg(l_dprice + r0 + k));
      if (atomicAdd(cnt + row[k], 1u) == 0u) atomicOr(kept + (key[k] >> 5), 1u << (key[k] & 31));
    }
  }
  for (int64_t i = (chunks << 3) + tid; i < n; i += stride) {
    if (l_shipdate[i] <= date_offset) continue;
    const int32_t key = l_orderkey[i];
    if (key < 0 || (int64_t)key >= n_map) continue;
    const int32_t row = key_to_row[key];
    if (row < 0 || (int64_t)row >= n_orders) continue;
    if (!((qual[row >> 5] >> (row & 31)) & 1u)) continue;
    atomicAdd(rev + row, (unsigned long long)(int64_t)l_dprice[i]);
    if (atomicAdd(cnt + row, 1u) == 0u) atomicOr(kept + (key >> 5), 1u << (key & 31));
  }
}

int grid_of(bo_ctx* ctx, int64_t items) {
  const int64_t need = (items + kQ3Block - 1) / kQ3Block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)ctx->num_sms * 8));
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q3(bo_ctx* ctx, const bo_tpch_q3_tables* t, int16_t date_offset, int32_t segment_code,
                          bo_tpch_q3_row* out_host, int64_t max_rows, int64_t* n_rows) {
  BO_CHECK_CTX(ctx);
  if (!t || !n_rows || max_rows < 0 || (max_rows > 0 && !out_host))
    return set_error(ctx, BO_ERR_INVALID, "q3: null argument");
  if (t->n_customer < 0 || t->n_orders < 0 || t->n_lineitem < 0 || t->n_orderkey_map < 0 || t->custkey_bound < 0)
    return set_error(ctx, BO_ERR_INVALID, "q3: negative size");
  if (t->n_orders > 0xffffffffll) return set_error(ctx, BO_ERR_INVALID, "q3: more than 2^32 orders");
  if ((t->n_customer > 0 && (!t->c_custkey || !t->c_mktsegment)) ||
      (t->n_orders > 0 && (!t->o_orderkey || !t->o_custkey || !t->o_orderdate)) ||
      (t->n_orderkey_map > 0 && !t->orderkey_to_row) ||
      (t->n_lineitem > 0 && (!t->l_orderkey || !t->l_shipdate || !t->l_discounted_price)))
    return set_error(ctx, BO_ERR_INVALID, "q3: null column");
  *n_rows = 0;
  const int64_t no = t->n_orders;
  if (no == 0 || segment_code < 0) return BO_OK;  // no order can qualify (unknown segment: none, :176-183)
  const int64_t mask_words = ((int64_t)t->custkey_bound + 31) / 32 + 1;
  const int64_t qual_words = (no + 31) / 32;
  size_t total = 0;
  auto add = [&](size_t b) { total += (b + 255) & ~size_t(255); };
  add(4 * (size_t)mask_words);
  add(4 * (size_t)qual_words);
  add(8 * (size_t)no);  // revenue
  add(4 * (size_t)no);  // count
  add(8 * (size_t)no);  // keys
  add(4 * (size_t)no);  // vals
  add(8 * (size_t)no);  // tmp keys
  add(4 * (size_t)no);  // tmp vals
  add(sizeof(bo_tpch_q3_row) * (size_t)no);
  const int64_t kept_words = t->n_orderkey_map / 32 + 1;
  const int64_t tiles = (kept_words + kBitmapTileWords - 1) / kBitmapTileWords;
  add(4 * (size_t)kept_words);                   // orderkeys with a counted lineitem
  add(4 * (size_t)std::max<int64_t>(tiles, 1));  // bitmap compaction's tile counts
  add(64);
  void* base = nullptr;
  int rc = region(ctx, "q3_ws", total, &base);
  if (rc) return rc;
  char* p = static_cast<char*>(base);
  uint32_t* mask = carve<uint32_t>(p, (size_t)mask_words);
  uint32_t* qual = carve<uint32_t>(p, (size_t)qual_words);
  unsigned long long* rev = carve<unsigned long long>(p, (size_t)no);
  uint32_t* cnt = carve<uint32_t>(p, (size_t)no);
  unsigned long long* keys = carve<unsigned long long>(p, (size_t)no);
  uint32_t* vals = carve<uint32_t>(p, (size_t)no);
  unsigned long long* tkeys = carve<unsigned long long>(p, (size_t)no);
  uint32_t* tvals = carve<uint32_t>(p, (size_t)no);
  bo_tpch_q3_row* rows = carve<bo_tpch_q3_row>(p, (size_t)no);
  uint32_t* kept = carve<uint32_t>(p, (size_t)kept_words);
  uint32_t* tile_counts = carve<uint32_t>(p, (size_t)std::max<int64_t>(tiles, 1));
  unsigned long long* n_out = carve<unsigned long long>(p, 8);
  // Scratch that accumulates starts at zero (the bitmaps are written whole or by atomicOr).
  BO_CUDA(ctx, cudaMemsetAsync(mask, 0, 4 * (size_t)mask_words, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(rev, 0, 8 * (size_t)no, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(cnt, 0, 4 * (size_t)no, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(kept, 0, 4 * (size_t)kept_words, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(n_out, 0, 16, ctx->stream));  // the count and the sort's overflow word
  if (t->n_customer > 0) {
    q3_cust_kernel<<<grid_of(ctx, t->n_customer), kQ3Block, 0, ctx->stream>>>(
        t->c_custkey, t->c_mktsegment, t->n_customer, segment_code, t->custkey_bound, mask);
    if ((rc = after_launch(ctx, "q3_cust_kernel"))) return rc;
  }
  q3_orders_kernel<<<grid_of(ctx, no), kQ3Block, 0, ctx->stream>>>(t->o_custkey, t->o_orderdate, no, date_offset,
                                                                     t->custkey_bound, mask, qual);
  if ((rc = after_launch(ctx, "q3_orders_kernel"))) return rc;
  if (t->n_lineitem > 0 && t->n_orderkey_map > 0) {
    if (aligned16(t->l_orderkey) && aligned16(t->l_shipdate)) {
      q3_lineitem_v8_kernel<<<grid_of(ctx, (t->n_lineitem + 7) / 8), kQ3Block, 0, ctx->stream>>>(
          t->l_orderkey, t->l_shipdate, t->l_discounted_price, t->n_lineitem, date_offset, t->orderkey_to_row,
          t->n_orderkey_map, no, qual, rev, cnt, kept);
      if ((rc = after_launch(ctx, "q3_lineitem_v8_kernel"))) return rc;
    } else {
      q3_lineitem_kernel<<<grid_of(ctx, t->n_lineitem), kQ3Block, 0, ctx->stream>>>(
          t->l_orderkey, t->l_shipdate, t->l_discounted_price, t->n_lineitem, date_offset, t->orderkey_to_row,
          t->n_orderkey_map, no, qual, rev, cnt, kept);
      if ((rc = after_launch(ctx, "q3_lineitem_kernel"))) return rc;
    }
  }
  // Qualifying orders in ascending orderkey order (no sort by orderkey
  // needed): the set bits of the kept bitmap (query_q3.cpp:348-355 breaks
  // ties by orderkey).
  if ((rc = bitmap_compact(ctx, kept, kept_words, tile_counts, vals, n_out))) return rc;
  // Sort keys and the sort itself without the result's size on the host: one
  // cluster launch reads the count on the device (up to 128K rows).  Rows go
  // straight into out_host when it is mapped pinned memory, so the query
  // synchronises once; a count beyond the cluster sets the overflow word and
  // the rows are sorted again with the count read back.
  uint32_t* overflow = reinterpret_cast<uint32_t*>(n_out + 1);
  q3_key2_kernel<<<grid_of(ctx, no), kQ3Block, 0, ctx->stream>>>(vals, t->orderkey_to_row, rev, t->o_orderdate, n_out,
                                                                  keys, ctx->d_err);
  if ((rc = after_launch(ctx, "q3_key2_kernel"))) return rc;
  if ((rc = cluster_sort_pairs_counted(ctx, keys, vals, n_out, no, 0, 64, overflow))) return rc;
  bo_tpch_q3_row* direct = nullptr;
  if (max_rows > 0) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, out_host) == cudaSuccess && attr.type == cudaMemoryTypeHost &&
        attr.devicePointer && aligned16(attr.devicePointer))
      direct = static_cast<bo_tpch_q3_row*>(attr.devicePointer);
    cudaGetLastError();  // pageable memory: not an error
  }
  auto gather = [&]() {
    const int64_t lim = direct ? std::min<int64_t>(max_rows, no) : no;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((lim + kQ3RowsBlock - 1) / kQ3RowsBlock,
                                                                 (int64_t)ctx->num_sms * 8));
    q3_gather_kernel<<<grid, kQ3RowsBlock, 0, ctx->stream>>>(vals, rev, t->o_orderkey, t->o_orderdate,
                                                             t->o_shippriority, n_out, lim, direct ? direct : rows);
    return after_launch(ctx, "q3_gather_kernel");
  };
  if ((rc = gather())) return rc;
  void* hs = nullptr;
  if ((rc = host_stage(ctx, 16, &hs))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(hs, n_out, 16, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // synchronises the stream
  if ((rc = device_error_status(ctx, bits, "q3"))) return rc;
  const unsigned long long nd = *static_cast<const unsigned long long*>(hs);
  const bool over = (*reinterpret_cast<const uint32_t*>(static_cast<const char*>(hs) + 8)) != 0u;
  const int64_t ns = (int64_t)std::min<unsigned long long>(nd, (unsigned long long)no);
  if (over) {  // more rows than one cluster sorts: the pass sequence, sized by the count now known
    if ((rc = radix_sort_pairs(ctx, keys, vals, tkeys, tvals, ns, 0, 64, nullptr))) return rc;
    if ((rc = gather())) return rc;
  }
  const int64_t m = std::min<int64_t>(ns, max_rows);
  if (!direct && m > 0)
    BO_CUDA(ctx, cudaMemcpyAsync(out_host, rows, sizeof(bo_tpch_q3_row) * (size_t)m, cudaMemcpyDeviceToHost,
                                 ctx->stream));
  if (over || (!direct && m > 0)) {
    if ((rc = consume_device_errors(ctx, &bits))) return rc;
    if ((rc = device_error_status(ctx, bits, "q3"))) return rc;
  }
  *n_rows = ns;
  return BO_OK;
}
