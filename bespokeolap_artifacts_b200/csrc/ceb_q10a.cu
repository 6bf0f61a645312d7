// CEB query 10a: run_q10a of bespoke_ceb/query_q10a.cpp:334-1130.
//
// The reference marks the titles of the allowed kinds (with their year),
// lists per title the dense indices of its movie_info values that pass the
// info-type and IN-list filters, collects the cast_info rows of those titles
// with an allowed role, keeps the persons whose name matches the ILIKE
// pattern, and aggregates MIN / MAX year per (name string, info value) --
// in a dense matrix when names x values fit kAggMaxSlots, else in a hash map.
// Here:
//   ceb_dim_mask_kernel        kind and role id masks;
//   q10a_title_kernel          present / has-year / year per title id;
//   q10a_info_kernel<false>    per-title counts of passing movie_info rows,
//   ceb_exclusive_scan         their offsets (exclusive scan, three launches),
//   q10a_info_kernel<true>     the rows' dense info indices scattered per title;
//   q10a_cast_kernel           (title, person) pairs of the allowed roles and
//                              the candidate persons (warp-aggregated appends);
//   q10a_name_match_kernel     ILIKE over the name dictionary, one thread per
//                              distinct name;
//   q10a_name_kernel           person -> name code for matching candidates;
//   q10a_agg_kernel<dense>     each pair times its title's info entries into the
//                              matrix (atomicMin / atomicMax) or the hash table;
//   q10a_emit_kernel           the used groups as result rows.
#include <algorithm>
#include <climits>
#include <vector>

#include "ceb.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr unsigned long long kEmptyKey = ~0ull;

struct Q10aMeta {
  unsigned int any_kind, any_role, n_pairs, n_rows;
  unsigned long long expansions;
  unsigned int bad;
};

__global__ void __launch_bounds__(kCebBlock) q10a_title_kernel(bo_ceb_q10a_tables t, const uint8_t* __restrict__ kind,
                                                               int32_t kind_size, int64_t title_bound,
                                                               uint8_t* __restrict__ present,
                                                               uint8_t* __restrict__ has_year,
                                                               int32_t* __restrict__ year) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < t.n_title; r += stride) {
    if (ceb_null(t.t_id, r) || ceb_null(t.t_kind_id, r)) continue;
    const int32_t k = t.t_kind_id.values[r], id = t.t_id.values[r];
    if (k < 0 || k >= kind_size || !kind[k] || id < 0 || (int64_t)id >= title_bound) continue;
    present[id] = 1;
    const bool yn = ceb_null(t.t_year, r);
    has_year[id] = yn ? 0 : 1;
    if (!yn) year[id] = t.t_year.values[r];
  }
}

// The movie_info rows the reference keeps (query_q10a.cpp:540-610): kScatter =
// false counts them per title, true writes their dense info index at the
// title's next position.
template <bool kScatter>
__global__ void __launch_bounds__(kCebBlock) q10a_info_kernel(bo_ceb_q10a_tables t,
                                                              const uint8_t* __restrict__ type_mask,
                                                              int32_t type_size, const int32_t* __restrict__ dense,
                                                              int32_t n_codes, const uint8_t* __restrict__ present,
                                                              int64_t title_bound, unsigned int* __restrict__ count,
                                                              const unsigned int* __restrict__ offset,
                                                              unsigned int* __restrict__ cursor,
                                                              int32_t* __restrict__ values) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < t.n_movie_info; r += stride) {
    if (ceb_null(t.mi_info_type_id, r) || ceb_null(t.mi_info, r)) continue;
    const int32_t ty = t.mi_info_type_id.values[r];
    if (ty < 0 || ty >= type_size || !type_mask[ty]) continue;
    const int32_t c = t.mi_info.values[r];
    if (c < 0 || c >= n_codes) continue;
    const int32_t d = dense[c];
    if (d < 0 || ceb_null(t.mi_movie_id, r)) continue;
    const int32_t m = t.mi_movie_id.values[r];
    if (m < 0 || (int64_t)m >= title_bound || !present[m]) continue;
    if (kScatter)
      values[offset[m] + atomicAdd(cursor + m, 1u)] = d;
    else
      atomicAdd(count + m, 1u);
  }
}

__global__ void __launch_bounds__(kCebBlock) q10a_cast_kernel(bo_ceb_q10a_tables t, const uint8_t* __restrict__ role,
                                                              int32_t role_size, const uint8_t* __restrict__ present,
                                                              const unsigned int* __restrict__ count,
                                                              int64_t title_bound, int64_t person_bound,
                                                              int2* __restrict__ pairs,
                                                              uint8_t* __restrict__ candidate,
                                                              Q10aMeta* __restrict__ meta) {
  unsigned long long exp = 0;
  const int64_t n = t.n_cast_info;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  const int64_t n_warp = (n + 31) & ~int64_t(31);
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < n_warp; r += stride) {
    bool take = false;
    int2 pr = make_int2(0, 0);
    if (r < n && !ceb_null(t.ci_movie_id, r) && !ceb_null(t.ci_role_id, r) && !ceb_null(t.ci_person_id, r)) {
      const int32_t m = t.ci_movie_id.values[r], ro = t.ci_role_id.values[r], p = t.ci_person_id.values[r];
      if (m >= 0 && (int64_t)m < title_bound && present[m] && count[m] && ro >= 0 && ro < role_size && role[ro] &&
          p >= 0 && (int64_t)p < person_bound) {
        take = true;
        pr = make_int2(m, p);
        candidate[p] = 1;
        exp += count[m];
      }
    }
    warp_append<int2>(take, pr, pairs, &meta->n_pairs);
  }
  for (int o = 16; o; o >>= 1) exp += __shfl_xor_sync(0xffffffffu, exp, o);
  if ((threadIdx.x & 31) == 0 && exp) atomicAdd(&meta->expansions, exp);
}

struct Pattern {
  int32_t type, len;
  const char* text;  // device
};

__global__ void __launch_bounds__(kCebBlock) q10a_name_match_kernel(const char* __restrict__ dict,
                                                                    const uint32_t* __restrict__ off, int64_t n_codes,
                                                                    Pattern pat, uint8_t* __restrict__ match) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t c = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; c < n_codes; c += stride) {
    const uint32_t b = off[c], e = off[c + 1];
    match[c] = ceb_like(pat.type, pat.text, pat.len, dict + b, (int)(e - b)) ? 1 : 0;
  }
}

__global__ void __launch_bounds__(kCebBlock) q10a_name_kernel(bo_ceb_q10a_tables t, const uint8_t* __restrict__ candidate,
                                                              int64_t person_bound, const uint8_t* __restrict__ match,
                                                              int32_t* __restrict__ person_name) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < t.n_name; r += stride) {
    if (ceb_null(t.nm_id, r) || ceb_null(t.nm_name, r)) continue;
    const int32_t p = t.nm_id.values[r], c = t.nm_name.values[r];
    if (p < 0 || (int64_t)p >= person_bound || !candidate[p] || c < 0 || (int64_t)c >= t.n_name_codes || !match[c])
      continue;
    person_name[p] = c;
  }
}

struct Agg {
  unsigned int* used;
  unsigned int* has;
  int* mn;
  int* mx;
  unsigned long long* keys;  // hash form
  unsigned long long mask;   // hash form: capacity - 1
};

__global__ void __launch_bounds__(kCebBlock) q10a_fill_kernel(Agg a, int64_t slots, bool hash) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t i = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; i < slots; i += stride) {
    a.used[i] = 0;
    a.has[i] = 0;
    a.mn[i] = INT_MAX;
    a.mx[i] = INT_MIN;
    if (hash) a.keys[i] = kEmptyKey;
  }
}

template <bool kDense>
__global__ void __launch_bounds__(kCebBlock) q10a_agg_kernel(const int2* __restrict__ pairs, Q10aMeta* __restrict__ meta,
                                                             const int32_t* __restrict__ person_name,
                                                             const unsigned int* __restrict__ offset,
                                                             const int32_t* __restrict__ values,
                                                             const uint8_t* __restrict__ has_year,
                                                             const int32_t* __restrict__ year, int32_t n_dense, Agg a) {
  const int64_t n = meta->n_pairs;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t i = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; i < n; i += stride) {
    const int2 pr = pairs[i];
    const int32_t name = person_name[pr.y];
    if (name < 0) continue;
    const bool hy = has_year[pr.x];
    const int32_t y = year[pr.x];
    for (unsigned int k = offset[pr.x]; k < offset[pr.x + 1]; ++k) {
      const int32_t d = values[k];
      unsigned long long slot;
      if (kDense) {
        slot = (unsigned long long)name * (unsigned long long)n_dense + (unsigned long long)d;
      } else {
        const unsigned long long key = ((unsigned long long)(uint32_t)name << 32) | (uint32_t)d;
        slot = (unsigned long long)hash32((uint32_t)name * 0x9e3779b9u ^ hash32((uint32_t)d)) & a.mask;
        unsigned long long probes = 0;
        for (;;) {
          const unsigned long long prev = atomicCAS(a.keys + slot, kEmptyKey, key);
          if (prev == kEmptyKey || prev == key) break;
          slot = (slot + 1) & a.mask;
          if (++probes > a.mask) {  // cannot happen at load <= 1/2; report rather than spin
            atomicOr(&meta->bad, 1u);
            break;
          }
        }
        if (probes > a.mask) continue;
      }
      if (!a.used[slot]) atomicOr(a.used + slot, 1u);
      if (hy) {
        if (!a.has[slot]) atomicOr(a.has + slot, 1u);
        atomicMin(a.mn + slot, y);
        atomicMax(a.mx + slot, y);
      }
    }
  }
}

__global__ void __launch_bounds__(kCebBlock) q10a_emit_kernel(Agg a, int64_t slots, bool hash, int32_t n_dense,
                                                              bo_ceb_q10a_row* __restrict__ rows, int64_t max_rows,
                                                              Q10aMeta* __restrict__ meta) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  const int64_t n_warp = (slots + 31) & ~int64_t(31);
  for (int64_t i = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; i < n_warp; i += stride) {
    bool take = false;
    bo_ceb_q10a_row row{};
    if (i < slots && a.used[i]) {
      take = true;
      if (hash) {
        const unsigned long long k = a.keys[i];
        row.name_code = (int32_t)(k >> 32);
        row.info_dense = (int32_t)(k & 0xffffffffu);
      } else {
        row.name_code = (int32_t)(i / n_dense);
        row.info_dense = (int32_t)(i % n_dense);
      }
      row.has_year = a.has[i] ? 1 : 0;
      row.min_year = row.has_year ? a.mn[i] : 0;
      row.max_year = row.has_year ? a.mx[i] : 0;
    }
    // Rows beyond max_rows are counted but not written.
    const unsigned int mask = __ballot_sync(0xffffffffu, take);
    if (!mask) continue;
    const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
    unsigned int base = 0;
    if (lane == leader) base = atomicAdd(&meta->n_rows, (unsigned int)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    const int64_t pos = (int64_t)base + __popc(mask & ((1u << lane) - 1u));
    if (take && pos < max_rows) rows[pos] = row;
  }
}

int q10a_grid(bo_ctx* ctx, const void* k, int64_t threads) {
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(k, kCebBlock, 0);
  return (int)std::max<int64_t>(1, std::min<int64_t>((threads + kCebBlock - 1) / kCebBlock, resident));
}

size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

bool col_ok(const bo_ceb_col& c, int64_t n) { return n == 0 || c.values; }

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_ceb_q10a(bo_ctx* ctx, const bo_ceb_q10a_tables* t, const bo_ceb_q10a_params* p,
                           bo_ceb_q10a_row* rows_out, int64_t max_rows, int64_t* n_rows_out, int32_t* dense_out) {
  BO_CHECK_CTX(ctx);
  if (!t || !p || !n_rows_out || max_rows < 0 || (max_rows > 0 && !rows_out))
    return set_error(ctx, BO_ERR_INVALID, "ceb_q10a: null argument");
  *n_rows_out = 0;
  if (dense_out) *dense_out = 0;
  const int64_t ns[] = {t->n_title, t->n_movie_info, t->n_cast_info, t->n_kind_type, t->n_role_type, t->n_name,
                        t->n_name_codes};
  for (int64_t n : ns)
    if (n < 0 || n > 0x7ffffffell) return set_error(ctx, BO_ERR_INVALID, "ceb_q10a: row count");
  if (p->info_type_size < 0 || p->n_info_codes < 0 || p->n_info_dense < 0 || p->n_kind_codes < 0 ||
      p->n_role_codes < 0 || p->pattern_len < 0 || p->pattern_type < kLikeAll || p->pattern_type > kLikeGeneral)
    return set_error(ctx, BO_ERR_INVALID, "ceb_q10a: parameter sizes");
  if (!col_ok(t->t_id, t->n_title) || !col_ok(t->t_kind_id, t->n_title) || !col_ok(t->t_year, t->n_title) ||
      !col_ok(t->mi_movie_id, t->n_movie_info) || !col_ok(t->mi_info_type_id, t->n_movie_info) ||
      !col_ok(t->mi_info, t->n_movie_info) || !col_ok(t->ci_movie_id, t->n_cast_info) ||
      !col_ok(t->ci_person_id, t->n_cast_info) || !col_ok(t->ci_role_id, t->n_cast_info) ||
      !col_ok(t->kt_id, t->n_kind_type) || !col_ok(t->kt_kind, t->n_kind_type) || !col_ok(t->rt_id, t->n_role_type) ||
      !col_ok(t->rt_role, t->n_role_type) || !col_ok(t->nm_id, t->n_name) || !col_ok(t->nm_name, t->n_name) ||
      (t->n_name_codes > 0 && !t->name_dict_offsets))
    return set_error(ctx, BO_ERR_INVALID, "ceb_q10a: null column");
  if ((p->info_type_size > 0 && !p->info_type_mask) || (p->n_info_codes > 0 && !p->info_dense) ||
      (p->n_kind_codes > 0 && !p->kind_allowed) || (p->n_role_codes > 0 && !p->role_allowed) ||
      (p->pattern_len > 0 && !p->pattern))
    return set_error(ctx, BO_ERR_INVALID, "ceb_q10a: null parameter array");
  if (t->n_title == 0 || t->n_movie_info == 0 || t->n_cast_info == 0 || t->n_name == 0 || p->n_info_dense == 0 ||
      t->n_name_codes == 0)
    return BO_OK;  // nothing can join: no rows (query_q10a.cpp:338-520 return early)
  const int64_t title_bound = t->n_title + 1, person_bound = t->n_name + 1;
  const int32_t kind_size = (int32_t)(t->n_kind_type + 1), role_size = (int32_t)(t->n_role_type + 1);
  // Workspace (everything before `zero_end` starts at zero).
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += al256(std::max<size_t>(bytes, 1));
    return o;
  };
  const size_t o_meta = take(sizeof(Q10aMeta));
  const size_t o_present = take((size_t)title_bound), o_hasy = take((size_t)title_bound);
  const size_t o_kind = take((size_t)kind_size), o_role = take((size_t)role_size);
  const size_t o_count = take(4 * (size_t)title_bound), o_cursor = take(4 * (size_t)title_bound);
  const size_t o_cand = take((size_t)person_bound);
  const size_t zero_end = off;
  const size_t o_year = take(4 * (size_t)title_bound);
  const size_t o_offset = take(4 * ((size_t)title_bound + 1));
  const size_t o_values = take(4 * (size_t)t->n_movie_info);
  const size_t o_pairs = take(sizeof(int2) * (size_t)t->n_cast_info);
  const size_t o_pname = take(4 * (size_t)person_bound);
  const size_t o_match = take((size_t)t->n_name_codes);
  const size_t o_tmask = take((size_t)p->info_type_size), o_dense = take(4 * (size_t)p->n_info_codes);
  const size_t o_ka = take((size_t)p->n_kind_codes), o_ra = take((size_t)p->n_role_codes);
  const size_t o_pat = take((size_t)p->pattern_len);
  void* wsp = nullptr;
  int rc = region(ctx, "ceb_q10a_ws", off, &wsp);
  if (rc) return rc;
  char* ws = static_cast<char*>(wsp);
  auto* meta = reinterpret_cast<Q10aMeta*>(ws + o_meta);
  auto* present = reinterpret_cast<uint8_t*>(ws + o_present);
  auto* hasy = reinterpret_cast<uint8_t*>(ws + o_hasy);
  auto* kind_mask = reinterpret_cast<uint8_t*>(ws + o_kind);
  auto* role_mask = reinterpret_cast<uint8_t*>(ws + o_role);
  auto* count = reinterpret_cast<unsigned int*>(ws + o_count);
  auto* cursor = reinterpret_cast<unsigned int*>(ws + o_cursor);
  auto* cand = reinterpret_cast<uint8_t*>(ws + o_cand);
  auto* year = reinterpret_cast<int32_t*>(ws + o_year);
  auto* offset = reinterpret_cast<unsigned int*>(ws + o_offset);
  auto* values = reinterpret_cast<int32_t*>(ws + o_values);
  auto* pairs = reinterpret_cast<int2*>(ws + o_pairs);
  auto* pname = reinterpret_cast<int32_t*>(ws + o_pname);
  auto* match = reinterpret_cast<uint8_t*>(ws + o_match);
  auto* tmask = reinterpret_cast<uint8_t*>(ws + o_tmask);
  auto* dense = reinterpret_cast<int32_t*>(ws + o_dense);
  auto *ka = reinterpret_cast<uint8_t*>(ws + o_ka), *ra = reinterpret_cast<uint8_t*>(ws + o_ra);
  auto* pat = reinterpret_cast<char*>(ws + o_pat);
  BO_CUDA(ctx, cudaMemsetAsync(ws, 0, zero_end, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(pname, 0xff, 4 * (size_t)person_bound, ctx->stream));  // -1: no name
  struct Copy {
    void* dst;
    const void* src;
    size_t n;
  } copies[] = {{tmask, p->info_type_mask, (size_t)p->info_type_size},
                {dense, p->info_dense, 4 * (size_t)p->n_info_codes},
                {ka, p->kind_allowed, (size_t)p->n_kind_codes},
                {ra, p->role_allowed, (size_t)p->n_role_codes},
                {pat, p->pattern, (size_t)p->pattern_len}};
  for (const auto& c : copies)
    if (c.n > 0) BO_CUDA(ctx, cudaMemcpyAsync(c.dst, c.src, c.n, cudaMemcpyHostToDevice, ctx->stream));
  const void* kd = reinterpret_cast<const void*>(&ceb_dim_mask_kernel);
  if (t->n_kind_type > 0) {
    ceb_dim_mask_kernel<<<q10a_grid(ctx, kd, t->n_kind_type), kCebBlock, 0, ctx->stream>>>(
        t->kt_id, t->kt_kind, t->n_kind_type, ka, p->n_kind_codes, kind_size, kind_mask, &meta->any_kind);
    if ((rc = after_launch(ctx, "ceb_dim_mask_kernel"))) return rc;
  }
  if (t->n_role_type > 0) {
    ceb_dim_mask_kernel<<<q10a_grid(ctx, kd, t->n_role_type), kCebBlock, 0, ctx->stream>>>(
        t->rt_id, t->rt_role, t->n_role_type, ra, p->n_role_codes, role_size, role_mask, &meta->any_role);
    if ((rc = after_launch(ctx, "ceb_dim_mask_kernel"))) return rc;
  }
  const void* kt = reinterpret_cast<const void*>(&q10a_title_kernel);
  q10a_title_kernel<<<q10a_grid(ctx, kt, t->n_title), kCebBlock, 0, ctx->stream>>>(*t, kind_mask, kind_size,
                                                                                  title_bound, present, hasy, year);
  if ((rc = after_launch(ctx, "q10a_title_kernel"))) return rc;
  const void* kc = reinterpret_cast<const void*>(&q10a_info_kernel<false>);
  const int gi = q10a_grid(ctx, kc, t->n_movie_info);
  q10a_info_kernel<false><<<gi, kCebBlock, 0, ctx->stream>>>(*t, tmask, p->info_type_size, dense, p->n_info_codes,
                                                             present, title_bound, count, nullptr, nullptr, nullptr);
  if ((rc = after_launch(ctx, "q10a_info_kernel"))) return rc;
  if ((rc = ceb_exclusive_scan(ctx, count, title_bound, offset))) return rc;
  q10a_info_kernel<true><<<gi, kCebBlock, 0, ctx->stream>>>(*t, tmask, p->info_type_size, dense, p->n_info_codes,
                                                            present, title_bound, nullptr, offset, cursor, values);
  if ((rc = after_launch(ctx, "q10a_info_kernel"))) return rc;
  const void* kk = reinterpret_cast<const void*>(&q10a_cast_kernel);
  q10a_cast_kernel<<<q10a_grid(ctx, kk, t->n_cast_info), kCebBlock, 0, ctx->stream>>>(
      *t, role_mask, role_size, present, count, title_bound, person_bound, pairs, cand, meta);
  if ((rc = after_launch(ctx, "q10a_cast_kernel"))) return rc;
  const void* km = reinterpret_cast<const void*>(&q10a_name_match_kernel);
  q10a_name_match_kernel<<<q10a_grid(ctx, km, t->n_name_codes), kCebBlock, 0, ctx->stream>>>(
      t->name_dict, t->name_dict_offsets, t->n_name_codes, Pattern{p->pattern_type, p->pattern_len, pat}, match);
  if ((rc = after_launch(ctx, "q10a_name_match_kernel"))) return rc;
  const void* kn = reinterpret_cast<const void*>(&q10a_name_kernel);
  q10a_name_kernel<<<q10a_grid(ctx, kn, t->n_name), kCebBlock, 0, ctx->stream>>>(*t, cand, person_bound, match,
                                                                                pname);
  if ((rc = after_launch(ctx, "q10a_name_kernel"))) return rc;
  // One host round trip: the pair count and the expansion bound size the
  // aggregation (matrix or hash table).
  Q10aMeta m{};
  BO_CUDA(ctx, cudaMemcpyAsync(&m, meta, sizeof(m), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (!m.any_kind || !m.any_role || m.n_pairs == 0) return BO_OK;
  const unsigned long long dense_slots = (unsigned long long)t->n_name_codes * (unsigned long long)p->n_info_dense;
  const bool use_dense = dense_slots <= (unsigned long long)BO_CEB_AGG_MAX_SLOTS;
  unsigned long long slots = dense_slots;
  if (!use_dense) {
    const unsigned long long groups = std::min<unsigned long long>(std::max<unsigned long long>(m.expansions, 1),
                                                                   dense_slots);
    slots = 1024;
    while (slots < 2 * groups) slots <<= 1;
  }
  const size_t agg_bytes = al256(4 * slots) * 4 + (use_dense ? 0 : al256(8 * slots)) +
                           al256(sizeof(bo_ceb_q10a_row) * (size_t)std::max<int64_t>(max_rows, 1));
  void* ap = nullptr;
  if ((rc = region(ctx, "ceb_q10a_agg", agg_bytes, &ap))) return rc;
  char* ab = static_cast<char*>(ap);
  Agg a{};
  a.used = reinterpret_cast<unsigned int*>(ab);
  a.has = reinterpret_cast<unsigned int*>(ab + al256(4 * slots));
  a.mn = reinterpret_cast<int*>(ab + 2 * al256(4 * slots));
  a.mx = reinterpret_cast<int*>(ab + 3 * al256(4 * slots));
  char* after = ab + 4 * al256(4 * slots);
  if (!use_dense) {
    a.keys = reinterpret_cast<unsigned long long*>(after);
    a.mask = slots - 1;
    after += al256(8 * slots);
  }
  auto* rows_dev = reinterpret_cast<bo_ceb_q10a_row*>(after);
  const void* kf = reinterpret_cast<const void*>(&q10a_fill_kernel);
  q10a_fill_kernel<<<q10a_grid(ctx, kf, (int64_t)slots), kCebBlock, 0, ctx->stream>>>(a, (int64_t)slots, !use_dense);
  if ((rc = after_launch(ctx, "q10a_fill_kernel"))) return rc;
  const void* ka2 = use_dense ? reinterpret_cast<const void*>(&q10a_agg_kernel<true>)
                              : reinterpret_cast<const void*>(&q10a_agg_kernel<false>);
  const int ga = q10a_grid(ctx, ka2, m.n_pairs);
  if (use_dense)
    q10a_agg_kernel<true><<<ga, kCebBlock, 0, ctx->stream>>>(pairs, meta, pname, offset, values, hasy, year,
                                                             p->n_info_dense, a);
  else
    q10a_agg_kernel<false><<<ga, kCebBlock, 0, ctx->stream>>>(pairs, meta, pname, offset, values, hasy, year,
                                                              p->n_info_dense, a);
  if ((rc = after_launch(ctx, "q10a_agg_kernel"))) return rc;
  const void* ke = reinterpret_cast<const void*>(&q10a_emit_kernel);
  q10a_emit_kernel<<<q10a_grid(ctx, ke, (int64_t)slots), kCebBlock, 0, ctx->stream>>>(
      a, (int64_t)slots, !use_dense, p->n_info_dense, rows_dev, max_rows, meta);
  if ((rc = after_launch(ctx, "q10a_emit_kernel"))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(&m, meta, sizeof(m), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (m.bad) return set_error(ctx, BO_ERR_OVERFLOW, "ceb_q10a: aggregation table full");
  *n_rows_out = m.n_rows;
  if (dense_out) *dense_out = use_dense ? 1 : 0;
  if ((int64_t)m.n_rows > max_rows)
    return set_error(ctx, BO_ERR_OVERFLOW, "ceb_q10a: %u groups, room for %lld", m.n_rows, (long long)max_rows);
  if (m.n_rows > 0) {
    BO_CUDA(ctx, cudaMemcpyAsync(rows_out, rows_dev, sizeof(bo_ceb_q10a_row) * m.n_rows, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return BO_OK;
}
