// TPC-H Q16 over the storage-plan layout: run_q16 of
// bespoke_tpch/query_q16.cpp:167-541, and the supplier complaint flags its
// supplier scan computes (:357-368, search :58-67).
//
// The reference assigns group ids in first-appearance order, collects
// (group, suppkey) entries, buckets them by group and counts distinct
// suppkeys with a stamp array, then sorts the groups by count descending and
// brand / type / size ascending.  Here a group is numbered by its sort
// position instead: g = (brand_rank * n_type + type_rank) * 64 + size, so
// ascending g is the tie order and one stable sort by count finishes it.
//   q16_part_kernel      qualifying part rows; each partkey keeps its last
//                        qualifying row's group (atomicMax of row << 32 | g)
//   q16_partsupp_kernel  partsupp rows of a grouped partkey and an unflagged
//                        supplier insert (g, suppkey) into a hash set; a new
//                        entry adds one to the group's count
//   ordered compaction   groups with a count, in g order
//   q16_keys_kernel      count-descending keys; one stable sort that reads
//                        the group count on the device
//   q16_rows_kernel      the rows, decoded from g
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "compact.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ16Block = 256;
constexpr int kQ16SizeBits = 6;        // sizes 0..50 below 64
constexpr uint32_t kQ16MaxSize = 50;   // run_q16's kMaxPartSize (:215-221)
constexpr int64_t kQ16MaxGroups = int64_t(1) << 28;
constexpr unsigned long long kEmpty = ~0ull;

struct Q16Dev {
  const uint16_t* brand_rank;
  const uint16_t* type_rank;
  const uint8_t* type_banned;
  const uint16_t* brand_of_rank;
  const uint16_t* type_of_rank;
};

__device__ __forceinline__ unsigned long long q16_hash(unsigned long long k) {
  k ^= k >> 31;
  k *= 0x7fb5d329728ea185ull;
  k ^= k >> 27;
  k *= 0x81dadef4bc2dd44dull;
  k ^= k >> 33;
  return k;
}

__global__ void __launch_bounds__(kQ16Block) q16_part_kernel(bo_tpch_q16_tables t, uint64_t size_mask,
                                                             int32_t banned_brand, int32_t n_brand, int32_t n_type,
                                                             Q16Dev d, unsigned long long* __restrict__ best,
                                                             uint32_t* err) {
  for (int64_t row = (int64_t)blockIdx.x * kQ16Block + threadIdx.x; row < t.n_part;
       row += (int64_t)gridDim.x * kQ16Block) {
    const int32_t b = t.p_brand[row];
    if (b == banned_brand) continue;
    const int32_t sz = t.p_size[row];
    if (sz < 0 || sz > (int32_t)kQ16MaxSize || !((size_mask >> sz) & 1ull)) continue;
    const int32_t ty = t.p_type[row];
    if (b >= n_brand || ty >= n_type) {
      raise_error(err, kErrBadGroupCode);
      continue;
    }
    if (d.type_banned[ty]) continue;
    const int32_t pk = t.p_partkey[row];
    if (pk < 0 || (int64_t)pk > t.n_part) continue;  // the reference's map holds keys 0..row_count
    const uint32_t g = (((uint32_t)d.brand_rank[b] * (uint32_t)n_type + d.type_rank[ty]) << kQ16SizeBits) | (uint32_t)sz;
    atomicMax(best + pk, ((unsigned long long)(row + 1) << 32) | g);
  }
}

__global__ void __launch_bounds__(kQ16Block) q16_partsupp_kernel(bo_tpch_q16_tables t, int32_t rows_per_part,
                                                                 const unsigned long long* __restrict__ best,
                                                                 unsigned long long* __restrict__ set,
                                                                 unsigned long long set_mask,
                                                                 uint32_t* __restrict__ cnt, uint32_t* err) {
  for (int64_t row = (int64_t)blockIdx.x * kQ16Block + threadIdx.x; row < t.n_partsupp;
       row += (int64_t)gridDim.x * kQ16Block) {
    const int64_t pk = rows_per_part > 0 ? row / rows_per_part + 1 : (int64_t)t.ps_partkey[row];
    if (pk < 0 || pk > t.n_part) continue;
    const unsigned long long b = __ldg(best + pk);
    if (!b) continue;
    const int32_t sk = t.ps_suppkey[row];
    if (sk < 0) continue;
    if ((int64_t)sk < t.n_banned && __ldg(t.s_banned + sk)) continue;
    const uint32_t g = (uint32_t)b;
    const unsigned long long key = ((unsigned long long)g << 32) | (uint32_t)sk;
    unsigned long long h = q16_hash(key) & set_mask;
    bool placed = false;
    for (unsigned long long probe = 0; probe <= set_mask; ++probe) {
      const unsigned long long prev = atomicCAS(set + h, kEmpty, key);
      if (prev == kEmpty) {
        atomicAdd(cnt + g, 1u);
        placed = true;
        break;
      }
      if (prev == key) {
        placed = true;
        break;
      }
      h = (h + 1) & set_mask;
    }
    if (!placed) raise_error(err, kErrTableOverflow);
  }
}

struct Q16Kept {
  const uint32_t* cnt;
  __device__ __forceinline__ bool operator()(int64_t g, uint32_t& v) const {
    if (__ldg(cnt + g) == 0u) return false;
    v = (uint32_t)g;
    return true;
  }
};

// The first min(*n_dev, limit) entries.
__device__ __forceinline__ int64_t q16_count(const unsigned long long* n_dev, int64_t limit) {
  const unsigned long long nd = *n_dev;
  return nd < (unsigned long long)limit ? (int64_t)nd : limit;
}

// keys[i] = max_count - count of group vals[i]: ascending keys are counts descending.
__global__ void __launch_bounds__(kQ16Block) q16_keys_kernel(const uint32_t* __restrict__ groups,
                                                             const uint32_t* __restrict__ cnt,
                                                             const unsigned long long* n_dev, int64_t limit,
                                                             uint32_t max_count, unsigned long long* __restrict__ keys) {
  const int64_t n = q16_count(n_dev, limit);
  for (int64_t i = (int64_t)blockIdx.x * kQ16Block + threadIdx.x; i < n; i += (int64_t)gridDim.x * kQ16Block)
    keys[i] = (unsigned long long)(max_count - cnt[groups[i]]);
}

__global__ void __launch_bounds__(kQ16Block) q16_rows_kernel(const uint32_t* __restrict__ groups,
                                                             const uint32_t* __restrict__ cnt,
                                                             const unsigned long long* n_dev, int64_t limit,
                                                             int32_t n_type, Q16Dev d, bo_tpch_q16_row* __restrict__ rows) {
  const int64_t n = q16_count(n_dev, limit);
  for (int64_t i = (int64_t)blockIdx.x * kQ16Block + threadIdx.x; i < n; i += (int64_t)gridDim.x * kQ16Block) {
    const uint32_t g = groups[i];
    const uint32_t bt = g >> kQ16SizeBits;
    bo_tpch_q16_row r;
    r.brand_code = d.brand_of_rank[bt / (uint32_t)n_type];
    r.type_code = d.type_of_rank[bt % (uint32_t)n_type];
    r.size = (int32_t)(g & ((1u << kQ16SizeBits) - 1));
    r.pad = 0;
    r.supplier_cnt = cnt[g];
    rows[i] = r;
  }
}

// One thread per supplier row: "Customer" somewhere, then "Complaints" at or
// after the byte following it (std::string_view::find semantics).
__device__ __forceinline__ bool has_at(const char* s, int64_t len, int64_t pos, const char* w, int wl) {
  if (pos + wl > len) return false;
  for (int j = 0; j < wl; ++j)
    if (s[pos + j] != w[j]) return false;
  return true;
}

__global__ void __launch_bounds__(kQ16Block) supplier_complaints_kernel(const char* __restrict__ comments,
                                                                        const uint32_t* __restrict__ offsets,
                                                                        const int32_t* __restrict__ suppkeys,
                                                                        int64_t n, uint8_t* __restrict__ banned,
                                                                        int64_t n_banned) {
  const char kCustomer[] = "Customer";
  const char kComplaints[] = "Complaints";
  for (int64_t r = (int64_t)blockIdx.x * kQ16Block + threadIdx.x; r < n; r += (int64_t)gridDim.x * kQ16Block) {
    const uint32_t b = offsets[r], e = offsets[r + 1];
    const char* s = comments + b;
    const int64_t len = e > b ? (int64_t)(e - b) : 0;
    int64_t at = -1;
    for (int64_t p = 0; p + 8 <= len && at < 0; ++p)
      if (has_at(s, len, p, kCustomer, 8)) at = p;
    if (at < 0) continue;
    bool hit = false;
    for (int64_t p = at + 8; p + 10 <= len && !hit; ++p) hit = has_at(s, len, p, kComplaints, 10);
    const int32_t k = suppkeys[r];
    if (hit && k >= 0 && (int64_t)k < n_banned) banned[k] = 1;
  }
}

int q16_grid(bo_ctx* ctx, int64_t items) {
  const int64_t need = (items + kQ16Block - 1) / kQ16Block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)ctx->num_sms * 8));
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_supplier_complaints(bo_ctx* ctx, const char* comments_device, const uint32_t* offsets_device,
                                           const int32_t* suppkeys_device, int64_t n_supplier, uint8_t* banned_out,
                                           int64_t n_banned) {
  BO_CHECK_CTX(ctx);
  if (n_supplier < 0 || n_banned < 0) return set_error(ctx, BO_ERR_INVALID, "supplier_complaints: negative size");
  if ((n_banned > 0 && !banned_out) || (n_supplier > 0 && (!offsets_device || !suppkeys_device)))
    return set_error(ctx, BO_ERR_INVALID, "supplier_complaints: null argument");
  if (n_banned > 0) BO_CUDA(ctx, cudaMemsetAsync(banned_out, 0, (size_t)n_banned, ctx->stream));
  if (n_supplier == 0 || n_banned == 0) return BO_OK;
  supplier_complaints_kernel<<<q16_grid(ctx, n_supplier), kQ16Block, 0, ctx->stream>>>(
      comments_device, offsets_device, suppkeys_device, n_supplier, banned_out, n_banned);
  return after_launch(ctx, "supplier_complaints_kernel");
}

extern "C" int bo_tpch_q16(bo_ctx* ctx, const bo_tpch_q16_tables* t, const bo_tpch_q16_params* prm,
                           bo_tpch_q16_row* rows_out, int64_t max_rows, int64_t* n_rows) {
  BO_CHECK_CTX(ctx);
  if (!t || !prm || !n_rows || max_rows < 0 || (max_rows > 0 && !rows_out))
    return set_error(ctx, BO_ERR_INVALID, "q16: null argument");
  *n_rows = 0;
  if (t->n_part < 0 || t->n_partsupp < 0 || t->n_banned < 0 || prm->n_brand < 0 || prm->n_type < 0 ||
      prm->rows_per_part < 0)
    return set_error(ctx, BO_ERR_INVALID, "q16: negative size");
  if (t->n_part >= 0x7fffffffll || t->n_partsupp >= 0xffffffffll)
    return set_error(ctx, BO_ERR_INVALID, "q16: too many rows");
  if ((t->n_part > 0 && (!t->p_partkey || !t->p_brand || !t->p_type || !t->p_size)) ||
      (t->n_partsupp > 0 && (!t->ps_suppkey || (prm->rows_per_part == 0 && !t->ps_partkey))) ||
      (t->n_banned > 0 && !t->s_banned) ||
      (prm->n_brand > 0 && !prm->brand_rank) || (prm->n_type > 0 && (!prm->type_rank || !prm->type_banned)))
    return set_error(ctx, BO_ERR_INVALID, "q16: null column");
  if (prm->rows_per_part > 0 && (int64_t)prm->rows_per_part * t->n_part != t->n_partsupp)
    return set_error(ctx, BO_ERR_INVALID, "q16: rows_per_part %d does not divide the partsupp rows",
                     (int)prm->rows_per_part);
  const int64_t nb = prm->n_brand, nt = prm->n_type;
  if (nb > 65536 || nt > 65536 || nb * nt * 64 > kQ16MaxGroups)
    return set_error(ctx, BO_ERR_INVALID, "q16: %lld x %lld brand / type groups", (long long)nb, (long long)nt);
  if (t->n_part == 0 || t->n_partsupp == 0 || nb == 0 || nt == 0 || (prm->size_mask & ((2ull << kQ16MaxSize) - 1)) == 0)
    return BO_OK;
  // Ranks and their inverses, checked to be permutations (the rows kernel decodes through them).
  std::vector<uint16_t> host_params((size_t)(2 * nb + 2 * nt));
  std::vector<uint8_t> seen_b((size_t)nb, 0), seen_t((size_t)nt, 0);
  for (int64_t i = 0; i < nb; ++i) {
    const uint16_t r = prm->brand_rank[i];
    if (r >= nb || seen_b[r]) return set_error(ctx, BO_ERR_INVALID, "q16: brand ranks are not a permutation");
    seen_b[r] = 1;
    host_params[(size_t)i] = r;
    host_params[(size_t)(nb + r)] = (uint16_t)i;
  }
  for (int64_t i = 0; i < nt; ++i) {
    const uint16_t r = prm->type_rank[i];
    if (r >= nt || seen_t[r]) return set_error(ctx, BO_ERR_INVALID, "q16: type ranks are not a permutation");
    seen_t[r] = 1;
    host_params[(size_t)(2 * nb + i)] = r;
    host_params[(size_t)(2 * nb + nt + r)] = (uint16_t)i;
  }
  const int64_t n_groups = nb * nt * 64;
  const int64_t max_out = std::min<int64_t>(n_groups, t->n_part);  // every group has a part row
  int64_t cap = 1024;
  while (cap < 2 * t->n_partsupp) cap <<= 1;
  const int64_t tiles = (n_groups + kCompactTile - 1) / kCompactTile;
  const size_t param_bytes = sizeof(uint16_t) * host_params.size() + (size_t)nt;
  size_t total = 0;
  auto add = [&](size_t b) { total += (b + 255) & ~size_t(255); };
  add(param_bytes);
  add(8 * (size_t)(t->n_part + 1));  // best row / group per partkey
  add(4 * (size_t)n_groups);         // counts
  add(8 * (size_t)cap);              // (group, suppkey) set
  add(4 * (size_t)tiles);
  add(4 * (size_t)max_out);          // groups, compacted
  add(8 * (size_t)max_out);          // sort keys
  add(8 * (size_t)max_out);          // sort scratch
  add(4 * (size_t)max_out);
  add(sizeof(bo_tpch_q16_row) * (size_t)max_out);
  add(64);
  void* base = nullptr;
  int rc = region(ctx, "q16_ws", total, &base);
  if (rc) return rc;
  char* p = static_cast<char*>(base);
  char* dparams = carve<char>(p, param_bytes);
  unsigned long long* best = carve<unsigned long long>(p, (size_t)(t->n_part + 1));
  uint32_t* cnt = carve<uint32_t>(p, (size_t)n_groups);
  unsigned long long* set = carve<unsigned long long>(p, (size_t)cap);
  uint32_t* tile_counts = carve<uint32_t>(p, (size_t)tiles);
  uint32_t* groups = carve<uint32_t>(p, (size_t)max_out);
  unsigned long long* keys = carve<unsigned long long>(p, (size_t)max_out);
  unsigned long long* tkeys = carve<unsigned long long>(p, (size_t)max_out);
  uint32_t* tvals = carve<uint32_t>(p, (size_t)max_out);
  bo_tpch_q16_row* rows = carve<bo_tpch_q16_row>(p, (size_t)max_out);
  unsigned long long* n_out = carve<unsigned long long>(p, 8);
  void* h = nullptr;
  if ((rc = host_stage(ctx, param_bytes, &h))) return rc;
  std::memcpy(h, host_params.data(), sizeof(uint16_t) * host_params.size());
  std::memcpy(static_cast<char*>(h) + sizeof(uint16_t) * host_params.size(), prm->type_banned, (size_t)nt);
  BO_CUDA(ctx, cudaMemcpyAsync(dparams, h, param_bytes, cudaMemcpyHostToDevice, ctx->stream));
  const uint16_t* dp = reinterpret_cast<const uint16_t*>(dparams);
  const Q16Dev d{dp, dp + 2 * nb, reinterpret_cast<const uint8_t*>(dp + 2 * nb + 2 * nt), dp + nb, dp + 2 * nb + nt};
  BO_CUDA(ctx, cudaMemsetAsync(best, 0, 8 * (size_t)(t->n_part + 1), ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(cnt, 0, 4 * (size_t)n_groups, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(set, 0xff, 8 * (size_t)cap, ctx->stream));
  q16_part_kernel<<<q16_grid(ctx, t->n_part), kQ16Block, 0, ctx->stream>>>(
      *t, prm->size_mask, prm->banned_brand, (int32_t)nb, (int32_t)nt, d, best, ctx->d_err);
  if ((rc = after_launch(ctx, "q16_part_kernel"))) return rc;
  q16_partsupp_kernel<<<q16_grid(ctx, t->n_partsupp), kQ16Block, 0, ctx->stream>>>(
      *t, prm->rows_per_part, best, set, (unsigned long long)(cap - 1), cnt, ctx->d_err);
  if ((rc = after_launch(ctx, "q16_partsupp_kernel"))) return rc;
  if ((rc = ordered_compact(ctx, Q16Kept{cnt}, n_groups, tile_counts, groups, n_out))) return rc;
  // The sort and the rows read the group count on the device; the rows go
  // straight into rows_out where it is mapped pinned memory, so the query
  // synchronises once (a count beyond one cluster sort: sorted again after
  // the read-back).
  uint32_t* overflow = reinterpret_cast<uint32_t*>(n_out + 1);
  BO_CUDA(ctx, cudaMemsetAsync(overflow, 0, 8, ctx->stream));
  const uint32_t max_count = (uint32_t)t->n_partsupp;
  int bits = 1;
  while (bits < 32 && (max_count >> bits) != 0u) ++bits;
  q16_keys_kernel<<<q16_grid(ctx, max_out), kQ16Block, 0, ctx->stream>>>(groups, cnt, n_out, max_out, max_count,
                                                                          keys);
  if ((rc = after_launch(ctx, "q16_keys_kernel"))) return rc;
  if ((rc = cluster_sort_pairs_counted(ctx, keys, groups, n_out, max_out, 0, bits, overflow))) return rc;
  bo_tpch_q16_row* direct = max_rows > 0 ? static_cast<bo_tpch_q16_row*>(mapped_device_ptr(rows_out)) : nullptr;
  const int64_t lim = direct ? std::min<int64_t>(max_rows, max_out) : max_out;
  auto emit_rows = [&]() {
    q16_rows_kernel<<<q16_grid(ctx, lim), kQ16Block, 0, ctx->stream>>>(groups, cnt, n_out, lim, (int32_t)nt, d,
                                                                        direct ? direct : rows);
    return after_launch(ctx, "q16_rows_kernel");
  };
  if ((rc = emit_rows())) return rc;
  int64_t ns = 0;
  bool over = false;
  if ((rc = read_counted(ctx, "q16", n_out, max_out, &ns, &over))) return rc;
  if (over) {
    if ((rc = radix_sort_pairs(ctx, keys, groups, tkeys, tvals, ns, 0, bits, nullptr))) return rc;
    if ((rc = emit_rows())) return rc;
  }
  const int64_t m = std::min<int64_t>(ns, max_rows);
  if (!direct && m > 0)
    BO_CUDA(ctx, cudaMemcpyAsync(rows_out, rows, sizeof(bo_tpch_q16_row) * (size_t)m, cudaMemcpyDeviceToHost,
                                 ctx->stream));
  if (over || (!direct && m > 0)) {
    uint32_t ebits = 0;
    if ((rc = consume_device_errors(ctx, &ebits))) return rc;
    if ((rc = device_error_status(ctx, ebits, "q16"))) return rc;
  }
  *n_rows = ns;
  return BO_OK;
}
