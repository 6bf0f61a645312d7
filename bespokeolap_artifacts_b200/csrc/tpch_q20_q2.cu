// TPC-H Q20 and Q2 over the storage-plan layout: run_q20 of
// bespoke_tpch/query_q20.cpp:338-676 and run_q2 of query_q2.cpp:146-430.
//
// Q20.  The reference sums lineitem quantities into a hash map keyed by
// (partkey, suppkey), probes it from each partsupp row and lists qualifying
// suppliers sorted by name.  Only pairs that some partsupp row looks up
// matter, so here each lineitem adds its quantity to the first partsupp row
// of its pair (found in its partkey's run of the partkey-sorted rows): a
// dense array with no hash table to clear.  The suppliers come out of an
// ordered compaction over the builder's name order, so no sort runs.
//   q20_color_kernel     partkeys whose name starts with COLOR (bitmap)
//   q20_lineitem_kernel  shipped in range, supplier nation, colored partkey
//   q20_partsupp_kernel  2 * 100 * availqty > sum -> the suppkey qualifies
//   ordered compaction   supplier rows in name order
//
// Q2.  One thread per part row finds the least supplycost among its
// partsupp rows with a supplier in the region and emits every row at that
// cost; one radix sort by (supplier rank, partkey) orders them, the supplier
// rank being the row's position in the builder's (acctbal desc, nation name,
// s_name, row) order.
#include <algorithm>
#include <climits>
#include <cstring>

#include "common.cuh"
#include "compact.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ20Block = 256;
constexpr int kQ20MaxColor = 256;

int q20_grid(bo_ctx* ctx, int64_t items) {
  const int64_t need = (items + kQ20Block - 1) / kQ20Block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)ctx->num_sms * 8));
}

__device__ __forceinline__ bool bit_set(const uint32_t* bits, int64_t k) {
  return (__ldg(bits + (k >> 5)) >> (k & 31)) & 1u;
}

struct ColorPrefix {
  char c[kQ20MaxColor];
  int32_t len;
};

__global__ void __launch_bounds__(kQ20Block) q20_color_kernel(bo_tpch_q20_tables t, ColorPrefix color,
                                                              uint32_t* __restrict__ bits) {
  for (int64_t row = (int64_t)blockIdx.x * kQ20Block + threadIdx.x; row < t.n_part;
       row += (int64_t)gridDim.x * kQ20Block) {
    const int32_t pk = t.p_partkey[row];
    if (pk < 0 || pk > t.max_partkey) continue;
    const uint32_t b = t.p_name_offsets[row], e = t.p_name_offsets[row + 1];
    if (e < b || (int64_t)(e - b) < color.len) continue;
    bool ok = true;
    for (int j = 0; j < color.len && ok; ++j) ok = t.p_name[b + j] == color.c[j];
    if (ok) atomicOr(bits + (pk >> 5), 1u << (pk & 31));
  }
}

// The first row of [begin, end) with suppkey sk, or -1.
__device__ __forceinline__ int64_t first_pair_row(const int32_t* __restrict__ ps_suppkey, int64_t begin,
                                                  int64_t end, int32_t sk) {
  for (int64_t r = begin; r < end; ++r)
    if (__ldg(ps_suppkey + r) == sk) return r;
  return -1;
}

__global__ void __launch_bounds__(kQ20Block) q20_lineitem_kernel(bo_tpch_q20_tables t, int32_t nation_key,
                                                                 int32_t start, int32_t end,
                                                                 const uint32_t* __restrict__ bits,
                                                                 unsigned long long* __restrict__ sum,
                                                                 uint32_t* __restrict__ hit) {
  const uint32_t span = (uint32_t)(end - start);
  for (int64_t row = (int64_t)blockIdx.x * kQ20Block + threadIdx.x; row < t.n_lineitem;
       row += (int64_t)gridDim.x * kQ20Block) {
    if ((uint32_t)((int32_t)t.l_shipdate[row] - start) >= span) continue;
    if ((int32_t)t.l_supp_nation[row] != nation_key) continue;
    const int32_t pk = t.l_partkey[row];
    if (pk < 0 || pk > t.max_partkey || !bit_set(bits, pk)) continue;
    if ((int64_t)pk >= t.n_ps_part_keys) continue;  // no partsupp row looks this pair up
    const int64_t f = first_pair_row(t.ps_suppkey, __ldg(t.ps_part_begin + pk), __ldg(t.ps_part_begin + pk + 1),
                                     t.l_suppkey[row]);
    if (f < 0) continue;
    atomicAdd(sum + f, (unsigned long long)(long long)t.l_quantity[row]);
    if (!__ldg(hit + f)) atomicOr(hit + f, 1u);
  }
}

__global__ void __launch_bounds__(kQ20Block) q20_partsupp_kernel(bo_tpch_q20_tables t, int32_t nation_key,
                                                                 const uint32_t* __restrict__ bits,
                                                                 const unsigned long long* __restrict__ sum,
                                                                 const uint32_t* __restrict__ hit,
                                                                 uint8_t* __restrict__ qualified) {
  for (int64_t row = (int64_t)blockIdx.x * kQ20Block + threadIdx.x; row < t.n_partsupp;
       row += (int64_t)gridDim.x * kQ20Block) {
    const int32_t pk = t.ps_partkey[row];
    if (pk < 0 || pk > t.max_partkey || !bit_set(bits, pk)) continue;
    const int32_t sk = t.ps_suppkey[row];
    if (sk < 0 || sk > t.max_suppkey || (int32_t)__ldg(t.s_nation_by_key + sk) != nation_key) continue;
    if ((int64_t)pk >= t.n_ps_part_keys) continue;
    const int64_t f = first_pair_row(t.ps_suppkey, __ldg(t.ps_part_begin + pk), row + 1, sk);
    if (f < 0 || !hit[f]) continue;
    const long long s = (long long)sum[f];
    if ((long long)t.ps_availqty[row] * 2 * 100 > s) qualified[sk] = 1;
  }
}

struct Q20Kept {
  const int32_t* row_by_name;
  const int32_t* suppkey;
  const int32_t* nationkey;
  const uint8_t* qualified;
  int32_t max_suppkey;
  int32_t nation_key;
  __device__ __forceinline__ bool operator()(int64_t r, uint32_t& v) const {
    const int32_t row = __ldg(row_by_name + r);
    const int32_t sk = __ldg(suppkey + row);
    if (sk < 0 || sk > max_suppkey || !__ldg(qualified + sk) || __ldg(nationkey + row) != nation_key) return false;
    v = (uint32_t)row;
    return true;
  }
};

// ---------------------------------------------------------------- Q2 ----
constexpr int kQ2Block = 256;

__global__ void __launch_bounds__(kQ2Block) q2_part_kernel(bo_tpch_q2_tables t, int32_t target_size,
                                                           const uint8_t* __restrict__ type_ok, int32_t n_type,
                                                           const uint8_t* __restrict__ nation_ok, int32_t n_nation,
                                                           int64_t cap, unsigned long long* __restrict__ n_out,
                                                           unsigned long long* __restrict__ keys,
                                                           uint32_t* __restrict__ vals, uint32_t* err) {
  for (int64_t p = (int64_t)blockIdx.x * kQ2Block + threadIdx.x; p < t.n_part; p += (int64_t)gridDim.x * kQ2Block) {
    if (t.p_size[p] != target_size) continue;
    const int32_t ty = t.p_type[p];
    if (ty >= n_type) {
      raise_error(err, kErrBadGroupCode);
      continue;
    }
    if (!type_ok[ty]) continue;
    const int64_t pk = p + 1;
    if (pk >= t.n_ps_part_keys) continue;
    const int64_t b = __ldg(t.ps_part_begin + pk), e = __ldg(t.ps_part_begin + pk + 1);
    auto supplier_ok = [&](int64_t r, uint32_t& srow) {
      srow = (uint32_t)(__ldg(t.ps_suppkey + r) - 1);
      if ((int64_t)srow >= t.n_supplier) return false;
      const int32_t ni = __ldg(t.s_nation_idx + srow);
      return ni >= 0 && ni < n_nation && nation_ok[ni];
    };
    int32_t min_cost = INT_MAX;
    uint32_t ties = 0;
    for (int64_t r = b; r < e; ++r) {
      uint32_t srow;
      if (!supplier_ok(r, srow)) continue;
      const int32_t c = __ldg(t.ps_supplycost + r);
      if (c < min_cost) {
        min_cost = c;
        ties = 1;
      } else if (c == min_cost) {
        ++ties;
      }
    }
    if (min_cost == INT_MAX || ties == 0) continue;
    unsigned long long pos = atomicAdd(n_out, (unsigned long long)ties);
    for (int64_t r = b; r < e; ++r) {
      uint32_t srow;
      if (!supplier_ok(r, srow) || __ldg(t.ps_supplycost + r) != min_cost) continue;
      if ((int64_t)pos < cap) {
        keys[pos] = ((unsigned long long)__ldg(t.s_rank + srow) << 32) | (uint32_t)pk;
        vals[pos] = srow;
      } else {
        raise_error(err, kErrOutputOverflow);
      }
      ++pos;
    }
  }
}

// The first min(*n_dev, limit) sorted pairs as rows.
__global__ void __launch_bounds__(kQ2Block) q2_rows_kernel(const unsigned long long* __restrict__ keys,
                                                           const uint32_t* __restrict__ vals,
                                                           const unsigned long long* n_dev, int64_t limit,
                                                           const uint16_t* __restrict__ p_mfgr,
                                                           bo_tpch_q2_row* __restrict__ rows) {
  const unsigned long long nd = *n_dev;
  const int64_t n = nd < (unsigned long long)limit ? (int64_t)nd : limit;
  for (int64_t i = (int64_t)blockIdx.x * kQ2Block + threadIdx.x; i < n; i += (int64_t)gridDim.x * kQ2Block) {
    const int32_t pk = (int32_t)(uint32_t)keys[i];
    bo_tpch_q2_row r;
    r.partkey = pk;
    r.supplier_row = (int32_t)vals[i];
    r.mfgr_code = p_mfgr[pk - 1];
    r.pad = 0;
    rows[i] = r;
  }
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q20(bo_ctx* ctx, const bo_tpch_q20_tables* t, const char* color, int32_t color_len,
                           int32_t nation_key, int16_t start_offset, int16_t end_offset, int32_t* rows_out,
                           int64_t max_rows, int64_t* n_rows) {
  BO_CHECK_CTX(ctx);
  if (!t || !n_rows || max_rows < 0 || (max_rows > 0 && !rows_out) || color_len < 0 || (color_len > 0 && !color))
    return set_error(ctx, BO_ERR_INVALID, "q20: null argument");
  *n_rows = 0;
  if (color_len > kQ20MaxColor) return set_error(ctx, BO_ERR_INVALID, "q20: COLOR longer than %d bytes", kQ20MaxColor);
  if (t->n_part < 0 || t->n_lineitem < 0 || t->n_partsupp < 0 || t->n_ps_part_keys < 0 || t->n_supplier < 0)
    return set_error(ctx, BO_ERR_INVALID, "q20: negative size");
  if (t->n_supplier >= 0x7fffffffll) return set_error(ctx, BO_ERR_INVALID, "q20: too many suppliers");
  if ((t->n_part > 0 && (!t->p_partkey || !t->p_name_offsets || !t->p_name)) ||
      (t->n_lineitem > 0 && (!t->l_shipdate || !t->l_partkey || !t->l_suppkey || !t->l_supp_nation || !t->l_quantity)) ||
      (t->n_partsupp > 0 && (!t->ps_partkey || !t->ps_suppkey || !t->ps_availqty)) ||
      (t->n_ps_part_keys > 0 && !t->ps_part_begin) ||
      (t->max_suppkey >= 0 && !t->s_nation_by_key) ||
      (t->n_supplier > 0 && (!t->s_suppkey || !t->s_nationkey || !t->s_row_by_name)))
    return set_error(ctx, BO_ERR_INVALID, "q20: null column");
  // :370-372: no part keys, no rows; without suppliers nothing qualifies.
  if (t->max_partkey < 0 || t->max_suppkey < 0 || t->n_supplier == 0) return BO_OK;
  const int64_t words = (int64_t)t->max_partkey / 32 + 1;
  const int64_t nq = (int64_t)t->max_suppkey + 1;
  const int64_t tiles = (t->n_supplier + kCompactTile - 1) / kCompactTile;
  size_t total = 0;
  auto add = [&](size_t b) { total += (b + 255) & ~size_t(255); };
  add(4 * (size_t)words);
  add(8 * (size_t)std::max<int64_t>(t->n_partsupp, 1));
  add(4 * (size_t)std::max<int64_t>(t->n_partsupp, 1));
  add((size_t)nq);
  add(4 * (size_t)tiles);
  add(4 * (size_t)t->n_supplier);
  add(64);
  void* base = nullptr;
  int rc = region(ctx, "q20_ws", total, &base);
  if (rc) return rc;
  char* p = static_cast<char*>(base);
  uint32_t* bits = carve<uint32_t>(p, (size_t)words);
  unsigned long long* sum = carve<unsigned long long>(p, (size_t)std::max<int64_t>(t->n_partsupp, 1));
  uint32_t* hit = carve<uint32_t>(p, (size_t)std::max<int64_t>(t->n_partsupp, 1));
  uint8_t* qualified = carve<uint8_t>(p, (size_t)nq);
  uint32_t* tile_counts = carve<uint32_t>(p, (size_t)tiles);
  uint32_t* out = carve<uint32_t>(p, (size_t)t->n_supplier);
  unsigned long long* n_out = carve<unsigned long long>(p, 8);
  // One clear of everything up to the sums' end, then the flags (the layout is contiguous).
  BO_CUDA(ctx, cudaMemsetAsync(base, 0, static_cast<size_t>(reinterpret_cast<char*>(tile_counts) -
                                                            static_cast<char*>(base)),
                               ctx->stream));
  ColorPrefix cp{};
  if (color_len > 0) std::memcpy(cp.c, color, (size_t)color_len);
  cp.len = color_len;
  if (t->n_part > 0) {
    q20_color_kernel<<<q20_grid(ctx, t->n_part), kQ20Block, 0, ctx->stream>>>(*t, cp, bits);
    if ((rc = after_launch(ctx, "q20_color_kernel"))) return rc;
  }
  if (t->n_lineitem > 0 && t->n_partsupp > 0) {
    q20_lineitem_kernel<<<q20_grid(ctx, t->n_lineitem), kQ20Block, 0, ctx->stream>>>(
        *t, nation_key, (int32_t)start_offset, (int32_t)end_offset, bits, sum, hit);
    if ((rc = after_launch(ctx, "q20_lineitem_kernel"))) return rc;
    q20_partsupp_kernel<<<q20_grid(ctx, t->n_partsupp), kQ20Block, 0, ctx->stream>>>(*t, nation_key, bits, sum, hit,
                                                                                     qualified);
    if ((rc = after_launch(ctx, "q20_partsupp_kernel"))) return rc;
  }
  if ((rc = ordered_compact(ctx,
                            Q20Kept{t->s_row_by_name, t->s_suppkey, t->s_nationkey, qualified, t->max_suppkey,
                                    nation_key},
                            t->n_supplier, tile_counts, out, n_out)))
    return rc;
  int64_t ns = 0;
  if ((rc = read_device_count(ctx, n_out, t->n_supplier, &ns))) return rc;
  const int64_t m = std::min<int64_t>(ns, max_rows);
  if (m > 0)
    BO_CUDA(ctx, cudaMemcpyAsync(rows_out, out, sizeof(int32_t) * (size_t)m, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t ebits = 0;
  if ((rc = consume_device_errors(ctx, &ebits))) return rc;  // synchronises the stream
  if ((rc = device_error_status(ctx, ebits, "q20"))) return rc;
  *n_rows = ns;
  return BO_OK;
}

extern "C" int bo_tpch_q2(bo_ctx* ctx, const bo_tpch_q2_tables* t, int32_t target_size, const uint8_t* type_ok_host,
                          int32_t n_type, const uint8_t* nation_ok_host, int32_t n_nation, bo_tpch_q2_row* rows_out,
                          int64_t max_rows, int64_t* n_rows) {
  BO_CHECK_CTX(ctx);
  if (!t || !n_rows || max_rows < 0 || (max_rows > 0 && !rows_out) || n_type < 0 || n_nation < 0 ||
      (n_type > 0 && !type_ok_host) || (n_nation > 0 && !nation_ok_host))
    return set_error(ctx, BO_ERR_INVALID, "q2: null argument");
  *n_rows = 0;
  if (t->n_part < 0 || t->n_partsupp < 0 || t->n_ps_part_keys < 0 || t->n_supplier < 0)
    return set_error(ctx, BO_ERR_INVALID, "q2: negative size");
  if (t->n_part >= 0x7fffffffll || t->n_supplier >= 0x7fffffffll || t->n_partsupp >= 0xffffffffll)
    return set_error(ctx, BO_ERR_INVALID, "q2: too many rows");
  if ((t->n_part > 0 && (!t->p_size || !t->p_type || !t->p_mfgr)) ||
      (t->n_partsupp > 0 && (!t->ps_suppkey || !t->ps_supplycost)) || (t->n_ps_part_keys > 0 && !t->ps_part_begin) ||
      (t->n_supplier > 0 && (!t->s_nation_idx || !t->s_rank)))
    return set_error(ctx, BO_ERR_INVALID, "q2: null column");
  if (t->n_part == 0 || t->n_partsupp == 0 || t->n_supplier == 0 || t->n_ps_part_keys == 0 || n_type == 0 ||
      n_nation == 0)
    return BO_OK;
  const int64_t cap = t->n_partsupp;  // at most one row per partsupp row
  size_t total = 0;
  auto add = [&](size_t b) { total += (b + 255) & ~size_t(255); };
  add((size_t)n_type + (size_t)n_nation);
  add(8 * (size_t)cap);
  add(4 * (size_t)cap);
  add(8 * (size_t)cap);
  add(4 * (size_t)cap);
  add(sizeof(bo_tpch_q2_row) * (size_t)cap);
  add(64);
  void* base = nullptr;
  int rc = region(ctx, "q2_ws", total, &base);
  if (rc) return rc;
  char* p = static_cast<char*>(base);
  uint8_t* masks = carve<uint8_t>(p, (size_t)n_type + (size_t)n_nation);
  unsigned long long* keys = carve<unsigned long long>(p, (size_t)cap);
  uint32_t* vals = carve<uint32_t>(p, (size_t)cap);
  unsigned long long* tkeys = carve<unsigned long long>(p, (size_t)cap);
  uint32_t* tvals = carve<uint32_t>(p, (size_t)cap);
  bo_tpch_q2_row* rows = carve<bo_tpch_q2_row>(p, (size_t)cap);
  unsigned long long* n_out = carve<unsigned long long>(p, 8);
  void* h = nullptr;
  if ((rc = host_stage(ctx, (size_t)n_type + (size_t)n_nation, &h))) return rc;
  std::memcpy(h, type_ok_host, (size_t)n_type);
  std::memcpy(static_cast<char*>(h) + n_type, nation_ok_host, (size_t)n_nation);
  BO_CUDA(ctx, cudaMemcpyAsync(masks, h, (size_t)n_type + (size_t)n_nation, cudaMemcpyHostToDevice, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(n_out, 0, 16, ctx->stream));  // the count and the sort's overflow word
  q2_part_kernel<<<q20_grid(ctx, t->n_part), kQ2Block, 0, ctx->stream>>>(*t, target_size, masks, n_type,
                                                                          masks + n_type, n_nation, cap, n_out, keys,
                                                                          vals, ctx->d_err);
  if ((rc = after_launch(ctx, "q2_part_kernel"))) return rc;
  // Sort and rows read the count on the device; rows into mapped rows_out
  // directly: one synchronisation (a count beyond one cluster sort is sorted
  // again after the read-back).
  uint32_t* overflow = reinterpret_cast<uint32_t*>(n_out + 1);
  int rank_bits = 1;
  while (rank_bits < 32 && ((uint64_t)(t->n_supplier - 1) >> rank_bits) != 0) ++rank_bits;
  // Keys are rank << 32 | partkey: the low word and the rank's bits.
  if ((rc = cluster_sort_pairs_counted(ctx, keys, vals, n_out, cap, 0, 32 + rank_bits, overflow))) return rc;
  bo_tpch_q2_row* direct = max_rows > 0 ? static_cast<bo_tpch_q2_row*>(mapped_device_ptr(rows_out)) : nullptr;
  const int64_t lim = direct ? std::min<int64_t>(max_rows, cap) : cap;
  auto emit_rows = [&]() {
    q2_rows_kernel<<<q20_grid(ctx, lim), kQ2Block, 0, ctx->stream>>>(keys, vals, n_out, lim, t->p_mfgr,
                                                                      direct ? direct : rows);
    return after_launch(ctx, "q2_rows_kernel");
  };
  if ((rc = emit_rows())) return rc;
  int64_t ns = 0;
  bool over = false;
  if ((rc = read_counted(ctx, "q2", n_out, cap, &ns, &over))) return rc;
  if (over) {
    if ((rc = radix_sort_pairs(ctx, keys, vals, tkeys, tvals, ns, 0, 32 + rank_bits, nullptr))) return rc;
    if ((rc = emit_rows())) return rc;
  }
  const int64_t m = std::min<int64_t>(ns, max_rows);
  if (!direct && m > 0)
    BO_CUDA(ctx, cudaMemcpyAsync(rows_out, rows, sizeof(bo_tpch_q2_row) * (size_t)m, cudaMemcpyDeviceToHost,
                                 ctx->stream));
  if (over || (!direct && m > 0)) {
    uint32_t ebits = 0;
    if ((rc = consume_device_errors(ctx, &ebits))) return rc;
    if ((rc = device_error_status(ctx, ebits, "q2"))) return rc;
  }
  *n_rows = ns;
  return BO_OK;
}
