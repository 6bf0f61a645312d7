// TPC-H Q9 over the storage-plan layout: run_q9 of
// bespoke_tpch/query_q9.cpp:130-447.
//
// The reference marks the parts whose name contains the color, lays the
// partsupp rows out as per-part slots (suppkey, supplycost), maps each
// orderkey to its order year and then walks every lineitem of a marked part:
// the slot with the lineitem's suppkey gives the supply cost, and
// discounted_price - supplycost * quantity / 100 is summed per (supplier
// nation, order year).  Here:
//   q9_part_kernel      one thread per part row, byte substring search of
//                       the color in its name -> bit per partkey;
//   q9_order_year_kernel  year offset per orderkey from the orderkey map and
//                       a per-date year table (no division on the device);
//   q9_lineitem_kernel  eight partkeys per thread from two 16-byte loads, bit
//                       test; rows of marked parts scan their partkey's
//                       partsupp range (sorted partsupp, the slots' order)
//                       and add into per-block shared totals, flushed with
//                       one 64-bit atomic per touched group.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ9Block = 256;
constexpr int kQ9Rows = 8;
constexpr int kQ9SharedGroups = 2048;
constexpr int kQ9MaxDates = 1 << 17;  // int16 date offsets span at most 65,536 days

__global__ void __launch_bounds__(kQ9Block) q9_part_kernel(const char* __restrict__ names,
                                                           const uint32_t* __restrict__ offsets,
                                                           const int32_t* __restrict__ partkey, int64_t n_part,
                                                           int64_t n_keys, const char* __restrict__ color,
                                                           int32_t color_len, uint32_t* __restrict__ part_ok) {
  const int64_t stride = (int64_t)gridDim.x * kQ9Block;
  for (int64_t i = (int64_t)blockIdx.x * kQ9Block + threadIdx.x; i < n_part; i += stride) {
    const int32_t pk = partkey[i];
    if (pk < 0 || (int64_t)pk >= n_keys) continue;  // query_q9.cpp:143-146
    const uint32_t b = offsets[i], e = offsets[i + 1];
    const uint32_t len = e - b;
    bool found = color_len == 0;
    if (!found && len >= (uint32_t)color_len) {
      const char* s = names + b;
      const uint32_t last = len - (uint32_t)color_len;
      for (uint32_t p = 0; p <= last && !found; ++p) {
        int32_t j = 0;
        while (j < color_len && s[p + j] == color[j]) ++j;
        found = j == color_len;
      }
    }
    if (found) atomicOr(part_ok + (pk >> 5), 1u << (pk & 31));
  }
}

__global__ void __launch_bounds__(kQ9Block) q9_order_year_kernel(const int32_t* __restrict__ orderkey_to_row,
                                                                 int64_t n_keys,
                                                                 const int16_t* __restrict__ orderdate,
                                                                 int64_t n_orders, int32_t min_date,
                                                                 const int16_t* __restrict__ year_by_date,
                                                                 int32_t n_dates, int32_t first_year,
                                                                 uint8_t* __restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * kQ9Block;
  for (int64_t k = (int64_t)blockIdx.x * kQ9Block + threadIdx.x; k < n_keys; k += stride) {
    const int32_t row = orderkey_to_row[k];
    uint8_t y = 255;
    if (row >= 0 && (int64_t)row < n_orders) {
      const int32_t d = (int32_t)orderdate[row] - min_date;
      if (d >= 0 && d < n_dates) y = (uint8_t)(year_by_date[d] - first_year);
    }
    out[k] = y;
  }
}

struct Q9Args {
  int32_t nation_bound;
  int32_t year_span;
  int32_t groups;
  int32_t shared_groups;  // groups kept in shared memory (all of them, or 0)
};

__device__ __forceinline__ void q9_row(const bo_tpch_q9_tables& t, int64_t r, int32_t pk, const Q9Args& a,
                                       unsigned long long* __restrict__ s_tot, uint32_t* __restrict__ s_used,
                                       unsigned long long* __restrict__ g_tot, uint32_t* __restrict__ g_used) {
  const int32_t sk = t.l_suppkey[r];
  const int32_t b = __ldg(t.ps_part_begin + pk), e = __ldg(t.ps_part_begin + pk + 1);
  int32_t cost = 0;
  bool matched = false;
  for (int32_t j = b; j < e; ++j) {
    if (__ldg(t.ps_suppkey + j) == sk) {
      cost = __ldg(t.ps_supplycost + j);
      matched = true;
      break;
    }
  }
  // The reference's four-slot path also tests the unfilled slots, whose
  // suppkey field reads as -1 and whose cost as 0 (query_q9.cpp:262-291).
  if (!matched && t.slots_per_part == 4 && e - b < 4 && sk == -1) matched = true;
  if (!matched) return;
  const int32_t nat = t.l_supp_nation[r];
  if (nat < 0 || nat >= a.nation_bound) return;
  const int32_t ok = t.l_orderkey[r];
  if (ok < 0 || (int64_t)ok >= t.n_orderkeys) return;
  const int32_t y = __ldg(t.o_year_by_key + ok);
  if (y >= a.year_span) return;
  const int64_t supply_cost = (int64_t)cost * (int64_t)t.l_quantity[r] / 100;
  const int64_t v = (int64_t)t.l_discounted_price[r] - supply_cost;
  const int g = nat * a.year_span + y;
  if (g < a.shared_groups) {
    atomicAdd(s_tot + g, (unsigned long long)v);
    atomicOr(s_used + (g >> 5), 1u << (g & 31));
  } else {
    atomicAdd(g_tot + g, (unsigned long long)v);
    atomicOr(g_used + (g >> 5), 1u << (g & 31));
  }
}

__global__ void __launch_bounds__(kQ9Block) q9_lineitem_kernel(bo_tpch_q9_tables t, Q9Args a,
                                                               const uint32_t* __restrict__ part_ok,
                                                               unsigned long long* __restrict__ g_tot,
                                                               uint32_t* __restrict__ g_used) {
  __shared__ unsigned long long s_tot[kQ9SharedGroups];
  __shared__ uint32_t s_used[kQ9SharedGroups / 32];
  for (int i = threadIdx.x; i < a.shared_groups; i += kQ9Block) s_tot[i] = 0;
  for (int i = threadIdx.x; i < (a.shared_groups + 31) / 32; i += kQ9Block) s_used[i] = 0;
  __syncthreads();
  const int64_t n = t.n_lineitem;
  const int64_t stride = (int64_t)gridDim.x * kQ9Block;
  for (int64_t g = (int64_t)blockIdx.x * kQ9Block + threadIdx.x; g * kQ9Rows < n; g += stride) {
    const int64_t r0 = g * kQ9Rows;
    int32_t pk[kQ9Rows];
    if (r0 + kQ9Rows <= n) {
      const int4 a0 = ld_stream_v4(t.l_partkey + r0), a1 = ld_stream_v4(t.l_partkey + r0 + 4);
      pk[0] = a0.x, pk[1] = a0.y, pk[2] = a0.z, pk[3] = a0.w;
      pk[4] = a1.x, pk[5] = a1.y, pk[6] = a1.z, pk[7] = a1.w;
    } else {
#pragma unroll
      for (int k = 0; k < kQ9Rows; ++k) pk[k] = r0 + k < n ? t.l_partkey[r0 + k] : -1;
    }
#pragma unroll
    for (int k = 0; k < kQ9Rows; ++k) {
      const int32_t p = pk[k];
      if (p < 0 || (int64_t)p >= t.n_part_keys) continue;
      if (!((__ldg(part_ok + (p >> 5)) >> (p & 31)) & 1u)) continue;
      q9_row(t, r0 + k, p, a, s_tot, s_used, g_tot, g_used);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < a.shared_groups; i += kQ9Block) {
    if ((s_used[i >> 5] >> (i & 31)) & 1u) {
      atomicAdd(g_tot + i, s_tot[i]);
      atomicOr(g_used + (i >> 5), 1u << (i & 31));
    }
  }
}

int q9_grid(bo_ctx* ctx, const void* k, int64_t threads) {
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(k, kQ9Block, 0);
  return (int)std::max<int64_t>(1, std::min<int64_t>((threads + kQ9Block - 1) / kQ9Block, resident));
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_order_years(bo_ctx* ctx, const int32_t* orderkey_to_row, int64_t n_keys,
                                   const int16_t* o_orderdate, int64_t n_orders, int16_t min_orderdate,
                                   const int16_t* year_by_date_host, int32_t n_dates, int32_t first_year,
                                   uint8_t* out_device) {
  BO_CHECK_CTX(ctx);
  if (n_keys < 0 || n_orders < 0 || n_dates < 0 || n_dates > kQ9MaxDates)
    return set_error(ctx, BO_ERR_INVALID, "order_years: sizes (at most %d dates)", kQ9MaxDates);
  if (n_keys == 0) return BO_OK;
  if (!orderkey_to_row || !out_device || (n_orders > 0 && !o_orderdate) || (n_dates > 0 && !year_by_date_host))
    return set_error(ctx, BO_ERR_INVALID, "order_years: null argument");
  for (int32_t i = 0; i < n_dates; ++i)
    if (year_by_date_host[i] - first_year < 0 || year_by_date_host[i] - first_year > 254)
      return set_error(ctx, BO_ERR_INVALID, "order_years: a year outside [first_year, first_year + 254]");
  void* p = nullptr;
  int rc = region(ctx, "q9_years", sizeof(int16_t) * (size_t)std::max(n_dates, 1), &p);
  if (rc) return rc;
  auto* tab = static_cast<int16_t*>(p);
  if (n_dates > 0)
    BO_CUDA(ctx, cudaMemcpyAsync(tab, year_by_date_host, sizeof(int16_t) * (size_t)n_dates, cudaMemcpyHostToDevice,
                                 ctx->stream));
  const void* k = reinterpret_cast<const void*>(&q9_order_year_kernel);
  q9_order_year_kernel<<<q9_grid(ctx, k, n_keys), kQ9Block, 0, ctx->stream>>>(
      orderkey_to_row, n_keys, o_orderdate, n_orders, min_orderdate, tab, n_dates, first_year, out_device);
  if ((rc = after_launch(ctx, "q9_order_year_kernel"))) return rc;
  // The year table is staged from pageable host memory: wait before returning.
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return BO_OK;
}

extern "C" int bo_tpch_q9(bo_ctx* ctx, const bo_tpch_q9_tables* t, const char* color, int32_t color_len,
                          int32_t nation_bound, int32_t year_span, int64_t* totals_out, uint8_t* used_out) {
  BO_CHECK_CTX(ctx);
  if (!t || (color_len > 0 && !color) || color_len < 0) return set_error(ctx, BO_ERR_INVALID, "q9: null argument");
  if (nation_bound < 0 || year_span < 0 || (int64_t)nation_bound * year_span > (1 << 24))
    return set_error(ctx, BO_ERR_INVALID, "q9: group domain %d x %d", nation_bound, year_span);
  const int32_t groups = nation_bound * year_span;
  if (groups > 0 && (!totals_out || !used_out)) return set_error(ctx, BO_ERR_INVALID, "q9: null output");
  for (int32_t i = 0; i < groups; ++i) {
    totals_out[i] = 0;
    used_out[i] = 0;
  }
  if (t->n_lineitem < 0 || t->n_part < 0 || t->n_part_keys < 0 || t->n_orderkeys < 0 || t->n_part_keys > 0x7fffffff)
    return set_error(ctx, BO_ERR_INVALID, "q9: sizes");
  if (groups == 0 || t->n_lineitem == 0 || t->n_part == 0 || t->n_part_keys == 0) return BO_OK;
  if (!t->l_partkey || !t->l_suppkey || !t->l_orderkey || !t->l_quantity || !t->l_discounted_price ||
      !t->l_supp_nation || !t->p_name_offsets || !t->p_partkey || !t->ps_part_begin || !t->o_year_by_key ||
      (t->n_orderkeys == 0) || !aligned16(t->l_partkey))
    return set_error(ctx, BO_ERR_INVALID, "q9: null column or partkeys not 16-byte aligned");
  const size_t bitmap_words = (size_t)((t->n_part_keys + 31) / 32);
  const size_t color_bytes = ((size_t)color_len + 255) & ~size_t(255);
  const size_t tot_bytes = sizeof(unsigned long long) * (size_t)groups;
  const size_t used_words = (size_t)(groups + 31) / 32;
  const size_t bytes = color_bytes + sizeof(uint32_t) * bitmap_words + 256 + tot_bytes + 256 + 4 * used_words + 256;
  void* p = nullptr;
  int rc = region(ctx, "q9_ws", bytes, &p);
  if (rc) return rc;
  char* base = static_cast<char*>(p);
  char* d_color = base;
  auto* part_ok = reinterpret_cast<uint32_t*>(base + color_bytes);
  auto* g_tot = reinterpret_cast<unsigned long long*>(
      base + ((color_bytes + sizeof(uint32_t) * bitmap_words + 255) & ~size_t(255)));
  auto* g_used = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(g_tot) + ((tot_bytes + 255) & ~size_t(255)));
  BO_CUDA(ctx, cudaMemsetAsync(part_ok, 0, bytes - color_bytes, ctx->stream));
  if (color_len > 0)
    BO_CUDA(ctx, cudaMemcpyAsync(d_color, color, (size_t)color_len, cudaMemcpyHostToDevice, ctx->stream));
  const void* kp = reinterpret_cast<const void*>(&q9_part_kernel);
  q9_part_kernel<<<q9_grid(ctx, kp, t->n_part), kQ9Block, 0, ctx->stream>>>(
      t->p_name, t->p_name_offsets, t->p_partkey, t->n_part, t->n_part_keys, d_color, color_len, part_ok);
  if ((rc = after_launch(ctx, "q9_part_kernel"))) return rc;
  Q9Args a{nation_bound, year_span, groups, groups <= kQ9SharedGroups ? groups : 0};
  const void* kl = reinterpret_cast<const void*>(&q9_lineitem_kernel);
  q9_lineitem_kernel<<<q9_grid(ctx, kl, (t->n_lineitem + kQ9Rows - 1) / kQ9Rows), kQ9Block, 0, ctx->stream>>>(
      *t, a, part_ok, g_tot, g_used);
  if ((rc = after_launch(ctx, "q9_lineitem_kernel"))) return rc;
  std::vector<uint32_t> used((size_t)used_words);
  BO_CUDA(ctx, cudaMemcpyAsync(totals_out, g_tot, tot_bytes, cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaMemcpyAsync(used.data(), g_used, 4 * used_words, cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int32_t i = 0; i < groups; ++i) used_out[i] = (uint8_t)((used[(size_t)i >> 5] >> (i & 31)) & 1u);
  return BO_OK;
}
