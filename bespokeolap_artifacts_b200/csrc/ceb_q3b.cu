// CEB query 3b: run_q3b of bespoke_ceb/query_q3b.cpp:728-1420.
//
// The reference builds, per movie, a map company -> row count (companies
// whose name matches), a keyword count and a map person -> cast row count
// (titles of an allowed kind that match, roles allowed), keeps the persons
// whose pcode matches, then for every movie adds keywords x cast x company
// to the group (title, name, company) and orders the groups by count desc
// and the three strings.  Here the per-movie maps are sorted runs:
//   masks / ILIKE        kind and role id masks; one thread per distinct
//                        company name, title and pcode string;
//   q3b_company_kernel   company id -> name code of matching companies;
//   q3b_mc_kernel        (movie, company) keys of matching companies, sorted
//                        (onesweep), run-length counted (flags + device
//                        scan), with per-movie ranges of the runs;
//   q3b_mk_kernel        keyword rows per movie with companies;
//   q3b_title_kernel     movie -> title code (candidate movies, allowed kind,
//                        matching title);
//   q3b_cast_kernel      (movie, person) keys of allowed roles, sorted and
//                        run-length counted like the companies;
//   q3b_name_kernel      person -> name code when the pcode matches;
//   q3b_join_kernel      each (movie, person) run times the movie's company
//                        runs into a hash table keyed by the three string
//                        codes (one 64-bit key);
//   ordering             two stable radix sorts: by the strings' ranks, then
//                        by the complemented count.
#include <algorithm>

#include "ceb.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr unsigned long long kQ3bEmpty = ~0ull;

struct Q3bMeta {
  unsigned long long n_mc, n_ci, expansions, n_rows;
  unsigned int any_kind, any_role, any_comp, bad;
};

__global__ void __launch_bounds__(kCebBlock) q3b_company_kernel(bo_ceb_q3b_tables t, const uint8_t* __restrict__ cmatch,
                                                                int32_t map_size, int32_t* __restrict__ name_of,
                                                                Q3bMeta* __restrict__ meta) {
  bool hit = false;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < t.n_company_name; r += stride) {
    if (ceb_null(t.cn_id, r) || ceb_null(t.cn_name, r)) continue;
    const int32_t id = t.cn_id.values[r], c = t.cn_name.values[r];
    if (id < 0 || id >= map_size || c < 0 || (int64_t)c >= t.company_dict.n || !cmatch[c]) continue;
    name_of[id] = c;
    hit = true;
  }
  if (__any_sync(0xffffffffu, hit) && (threadIdx.x & 31) == 0) atomicOr(&meta->any_comp, 1u);
}

__global__ void __launch_bounds__(kCebBlock) q3b_mc_kernel(bo_ceb_q3b_tables t, const int32_t* __restrict__ name_of,
                                                           int32_t map_size, unsigned long long* __restrict__ keys,
                                                           Q3bMeta* __restrict__ meta) {
  const int64_t n = t.n_movie_companies;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  const int64_t n_warp = (n + 31) & ~int64_t(31);
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < n_warp; r += stride) {
    bool take = false;
    unsigned long long key = 0;
    if (r < n && !ceb_null(t.mc_movie_id, r) && !ceb_null(t.mc_company_id, r) &&
        !ceb_null(t.mc_company_type_id, r)) {
      const int32_t m = t.mc_movie_id.values[r], c = t.mc_company_id.values[r];
      if (m >= 0 && m < t.movie_bound && c >= 0 && c < map_size && name_of[c] >= 0) {
        take = true;
        key = ((unsigned long long)(uint32_t)m << 32) | (uint32_t)c;
      }
    }
    warp_append<unsigned long long, unsigned long long>(take, key, keys, &meta->n_mc);
  }
}

// Run-length counting of sorted keys: flags of run starts ...
__global__ void __launch_bounds__(kCebBlock) q3b_run_flag_kernel(const unsigned long long* __restrict__ keys,
                                                                 const unsigned long long* __restrict__ n_dev,
                                                                 int64_t n_max, unsigned int* __restrict__ flag) {
  const int64_t n = (int64_t)*n_dev;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t i = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; i < n_max; i += stride)
    flag[i] = (i < n && (i == 0 || keys[i] != keys[i - 1])) ? 1u : 0u;
}

// ... then each run's key, first row and length; per-movie ranges of runs.
__global__ void __launch_bounds__(kCebBlock) q3b_run_kernel(const unsigned long long* __restrict__ keys,
                                                            const unsigned long long* __restrict__ n_dev, int64_t n_max,
                                                            const unsigned int* __restrict__ flag,
                                                            const unsigned int* __restrict__ pos,
                                                            unsigned long long* __restrict__ run_key,
                                                            unsigned int* __restrict__ run_start) {
  const int64_t n = (int64_t)*n_dev;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t i = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; i < n; i += stride) {
    if (!flag[i]) continue;
    run_key[pos[i]] = keys[i];
    run_start[pos[i]] = (unsigned int)i;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) run_start[pos[n_max]] = (unsigned int)n;  // end of the last run
}

__global__ void __launch_bounds__(kCebBlock) q3b_movie_range_kernel(const unsigned long long* __restrict__ run_key,
                                                                    const unsigned int* __restrict__ n_runs_dev,
                                                                    unsigned int* __restrict__ begin,
                                                                    unsigned int* __restrict__ end,
                                                                    uint8_t* __restrict__ present) {
  const int64_t n = *n_runs_dev;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t j = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; j < n; j += stride) {
    const uint32_t m = (uint32_t)(run_key[j] >> 32);
    if (j == 0 || (uint32_t)(run_key[j - 1] >> 32) != m) {
      begin[m] = (unsigned int)j;
      if (present) present[m] = 1;
    }
    if (j == n - 1 || (uint32_t)(run_key[j + 1] >> 32) != m) end[m] = (unsigned int)j + 1;
  }
}

__global__ void __launch_bounds__(kCebBlock) q3b_mk_kernel(bo_ceb_q3b_tables t, const uint8_t* __restrict__ in_mc,
                                                           unsigned int* __restrict__ mk) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < t.n_movie_keyword; r += stride) {
    if (ceb_null(t.mk_movie_id, r) || ceb_null(t.mk_keyword_id, r)) continue;
    const int32_t m = t.mk_movie_id.values[r];
    if (m < 0 || m >= t.movie_bound || !in_mc[m]) continue;
    atomicAdd(mk + m, 1u);
  }
}

__global__ void __launch_bounds__(kCebBlock) q3b_title_kernel(bo_ceb_q3b_tables t, const uint8_t* __restrict__ in_mc,
                                                              const unsigned int* __restrict__ mk,
                                                              const uint8_t* __restrict__ kind_mask, int32_t kind_size,
                                                              const uint8_t* __restrict__ tmatch,
                                                              int32_t* __restrict__ title_of) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < t.n_title; r += stride) {
    if (ceb_null(t.t_id, r) || ceb_null(t.t_title, r) || ceb_null(t.t_kind_id, r)) continue;
    const int32_t m = t.t_id.values[r], k = t.t_kind_id.values[r], c = t.t_title.values[r];
    if (m < 0 || m >= t.movie_bound || !in_mc[m] || !mk[m]) continue;
    if (k < 0 || k >= kind_size || !kind_mask[k] || c < 0 || (int64_t)c >= t.title_dict.n || !tmatch[c]) continue;
    title_of[m] = c;
  }
}

__global__ void __launch_bounds__(kCebBlock) q3b_cast_kernel(bo_ceb_q3b_tables t, const int32_t* __restrict__ title_of,
                                                             const uint8_t* __restrict__ role_mask, int32_t role_size,
                                                             unsigned long long* __restrict__ keys,
                                                             uint8_t* __restrict__ cand, Q3bMeta* __restrict__ meta) {
  const int64_t n = t.n_cast_info;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  const int64_t n_warp = (n + 31) & ~int64_t(31);
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < n_warp; r += stride) {
    bool take = false;
    unsigned long long key = 0;
    if (r < n && !ceb_null(t.ci_movie_id, r) && !ceb_null(t.ci_person_id, r) && !ceb_null(t.ci_role_id, r)) {
      const int32_t m = t.ci_movie_id.values[r], p = t.ci_person_id.values[r], ro = t.ci_role_id.values[r];
      if (m >= 0 && m < t.movie_bound && title_of[m] >= 0 && ro >= 0 && ro < role_size && role_mask[ro]) {
        take = true;
        key = ((unsigned long long)(uint32_t)m << 32) | (uint32_t)p;
        if (p >= 0 && p < t.person_bound) cand[p] = 1;
      }
    }
    warp_append<unsigned long long, unsigned long long>(take, key, keys, &meta->n_ci);
  }
}

__global__ void __launch_bounds__(kCebBlock) q3b_name_kernel(bo_ceb_q3b_tables t, const uint8_t* __restrict__ cand,
                                                             const uint8_t* __restrict__ pmatch,
                                                             int32_t* __restrict__ name_of) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < t.n_name; r += stride) {
    if (ceb_null(t.nm_id, r) || ceb_null(t.nm_name, r) || ceb_null(t.nm_pcode, r)) continue;
    const int32_t p = t.nm_id.values[r], pc = t.nm_pcode.values[r];
    if (p < 0 || p >= t.person_bound || !cand[p] || pc < 0 || (int64_t)pc >= t.pcode_dict.n || !pmatch[pc]) continue;
    name_of[p] = t.nm_name.values[r];
  }
}

struct Runs {
  const unsigned long long* key;
  const unsigned int* start;  // n_runs + 1 entries
  const unsigned int* n;      // device run count
};

struct Pack {
  int nb, cb;  // bits of the name and company codes
};

__device__ __forceinline__ unsigned long long q3b_pack(const Pack& pk, uint32_t t, uint32_t n, uint32_t c) {
  return ((unsigned long long)t << (pk.nb + pk.cb)) | ((unsigned long long)n << pk.cb) | c;
}

// kJoin = false: the number of (person run, company run) combinations, to
// size the table; true: add keywords x cast x company to each group.
template <bool kJoin>
__global__ void __launch_bounds__(kCebBlock) q3b_join_kernel(Runs ci, Runs mc, const unsigned int* __restrict__ mc_begin,
                                                             const unsigned int* __restrict__ mc_end,
                                                             const unsigned int* __restrict__ mk,
                                                             const int32_t* __restrict__ title_of,
                                                             const int32_t* __restrict__ person_name,
                                                             const int32_t* __restrict__ company_name,
                                                             int32_t person_bound, Pack pk,
                                                             unsigned long long* __restrict__ hkeys,
                                                             unsigned long long* __restrict__ hcount,
                                                             unsigned long long hmask, Q3bMeta* __restrict__ meta) {
  const int64_t n = *ci.n;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  unsigned long long exp = 0;
  for (int64_t j = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; j < n; j += stride) {
    const unsigned long long k = ci.key[j];
    const uint32_t m = (uint32_t)(k >> 32);
    const int32_t p = (int32_t)(uint32_t)k;
    if (p < 0 || p >= person_bound) continue;
    const int32_t nm = person_name[p];
    if (nm < 0) continue;
    const unsigned int b = mc_begin[m], e = mc_end[m];
    if (!kJoin) {
      exp += e - b;
      continue;
    }
    const unsigned long long cnt = (unsigned long long)(ci.start[j + 1] - ci.start[j]) * mk[m];
    const uint32_t tc = (uint32_t)title_of[m];
    for (unsigned int q = b; q < e; ++q) {
      const int32_t cn = company_name[(uint32_t)mc.key[q]];
      const unsigned long long v = cnt * (unsigned long long)(mc.start[q + 1] - mc.start[q]);
      const unsigned long long key = q3b_pack(pk, tc, (uint32_t)nm, (uint32_t)cn);
      unsigned long long slot = (hash32((uint32_t)key ^ hash32((uint32_t)(key >> 32))) * 0x9e3779b97f4a7c15ull) &
                                hmask;
      unsigned long long probes = 0;
      for (;;) {
        const unsigned long long prev = atomicCAS(hkeys + slot, kQ3bEmpty, key);
        if (prev == kQ3bEmpty || prev == key) break;
        slot = (slot + 1) & hmask;
        if (++probes > hmask) break;
      }
      if (probes > hmask) {  // cannot happen at load <= 1/2; reported, never a spin
        atomicOr(&meta->bad, 1u);
        continue;
      }
      atomicAdd(hcount + slot, v);
    }
  }
  if (!kJoin) {
    for (int o = 16; o; o >>= 1) exp += __shfl_xor_sync(0xffffffffu, exp, o);
    if ((threadIdx.x & 31) == 0 && exp) atomicAdd(&meta->expansions, exp);
  }
}

__global__ void __launch_bounds__(kCebBlock) q3b_emit_kernel(const unsigned long long* __restrict__ hkeys,
                                                             const unsigned long long* __restrict__ hcount,
                                                             unsigned long long slots,
                                                             unsigned long long* __restrict__ out_key,
                                                             unsigned long long* __restrict__ out_count,
                                                             Q3bMeta* __restrict__ meta) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  const int64_t n_warp = ((int64_t)slots + 31) & ~int64_t(31);
  for (int64_t i = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; i < n_warp; i += stride) {
    const bool take = i < (int64_t)slots && hkeys[i] != kQ3bEmpty;
    const unsigned int mask = __ballot_sync(0xffffffffu, take);
    if (!mask) continue;
    const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(&meta->n_rows, (unsigned long long)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (take) {
      const unsigned long long pos = base + __popc(mask & ((1u << lane) - 1u));
      out_key[pos] = hkeys[i];
      out_count[pos] = hcount[i];
    }
  }
}

// Sort keys: the strings' ranks packed like the codes (pass 1), then the
// complemented counts of the rows in that order (pass 2).
__global__ void __launch_bounds__(kCebBlock) q3b_rank_key_kernel(const unsigned long long* __restrict__ key,
                                                                 int64_t n, Pack pk, const int32_t* __restrict__ trank,
                                                                 const int32_t* __restrict__ nrank,
                                                                 const int32_t* __restrict__ crank,
                                                                 unsigned long long* __restrict__ sk,
                                                                 uint32_t* __restrict__ idx) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  const unsigned long long nmask = (1ull << pk.nb) - 1, cmask = (1ull << pk.cb) - 1;
  for (int64_t i = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; i < n; i += stride) {
    const unsigned long long k = key[i];
    const uint32_t t = (uint32_t)(k >> (pk.nb + pk.cb)), nm = (uint32_t)((k >> pk.cb) & nmask),
                   c = (uint32_t)(k & cmask);
    sk[i] = q3b_pack(pk, (uint32_t)trank[t], (uint32_t)nrank[nm], (uint32_t)crank[c]);
    idx[i] = (uint32_t)i;
  }
}

__global__ void __launch_bounds__(kCebBlock) q3b_count_key_kernel(const unsigned long long* __restrict__ count,
                                                                  const uint32_t* __restrict__ idx, int64_t n,
                                                                  unsigned long long* __restrict__ sk) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t i = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; i < n; i += stride) sk[i] = ~count[idx[i]];
}

__global__ void __launch_bounds__(kCebBlock) q3b_rows_kernel(const unsigned long long* __restrict__ key,
                                                             const unsigned long long* __restrict__ count,
                                                             const uint32_t* __restrict__ idx, int64_t n, Pack pk,
                                                             bo_ceb_q3b_row* __restrict__ rows) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  const unsigned long long nmask = (1ull << pk.nb) - 1, cmask = (1ull << pk.cb) - 1;
  for (int64_t i = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; i < n; i += stride) {
    const uint32_t s = idx[i];
    const unsigned long long k = key[s];
    bo_ceb_q3b_row r;
    r.title_code = (int32_t)(k >> (pk.nb + pk.cb));
    r.name_code = (int32_t)((k >> pk.cb) & nmask);
    r.company_code = (int32_t)(k & cmask);
    r.pad = 0;
    r.count = (int64_t)count[s];
    rows[i] = r;
  }
}

int q3b_grid(bo_ctx* ctx, const void* k, int64_t threads) {
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(k, kCebBlock, 0);
  return (int)std::max<int64_t>(1, std::min<int64_t>((threads + kCebBlock - 1) / kCebBlock, resident));
}

size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

int bits_for(int64_t n) {
  int b = 1;
  while (b < 62 && (1ll << b) < n) ++b;
  return b;
}

bool col_ok(const bo_ceb_col& c, int64_t n) { return n == 0 || c.values; }

// Sorted runs of the n_dev keys in keys[0 .. n_max): run keys, run starts
// (n_runs + 1 entries) and the device run count (runs_n).
int q3b_runs(bo_ctx* ctx, unsigned long long* keys, uint32_t* vals, unsigned long long* tmp_keys, uint32_t* tmp_vals,
             int64_t n_max, const unsigned long long* n_dev, unsigned int* flag, unsigned int* pos,
             unsigned long long* run_key, unsigned int* run_start) {
  int rc = radix_sort_pairs(ctx, keys, vals, tmp_keys, tmp_vals, n_max, 0, 64, n_dev);
  if (rc) return rc;
  const void* kf = reinterpret_cast<const void*>(&q3b_run_flag_kernel);
  q3b_run_flag_kernel<<<q3b_grid(ctx, kf, n_max), kCebBlock, 0, ctx->stream>>>(keys, n_dev, n_max, flag);
  if ((rc = after_launch(ctx, "q3b_run_flag_kernel"))) return rc;
  if ((rc = ceb_exclusive_scan(ctx, flag, n_max, pos))) return rc;
  const void* kr = reinterpret_cast<const void*>(&q3b_run_kernel);
  q3b_run_kernel<<<q3b_grid(ctx, kr, n_max), kCebBlock, 0, ctx->stream>>>(keys, n_dev, n_max, flag, pos, run_key,
                                                                          run_start);
  return after_launch(ctx, "q3b_run_kernel");
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_ceb_q3b(bo_ctx* ctx, const bo_ceb_q3b_tables* t, const bo_ceb_q3b_params* p,
                          bo_ceb_q3b_row* rows_out, int64_t max_rows, int64_t* n_rows_out) {
  BO_CHECK_CTX(ctx);
  if (!t || !p || !n_rows_out || max_rows < 0 || (max_rows > 0 && !rows_out))
    return set_error(ctx, BO_ERR_INVALID, "ceb_q3b: null argument");
  *n_rows_out = 0;
  const int64_t ns[] = {t->n_kind_type, t->n_role_type, t->n_company_name, t->n_movie_companies, t->n_movie_keyword,
                        t->n_title, t->n_cast_info, t->n_name, t->title_dict.n, t->name_dict.n, t->company_dict.n,
                        t->pcode_dict.n};
  for (int64_t n : ns)
    if (n < 0 || n > 0x7ffffffell) return set_error(ctx, BO_ERR_INVALID, "ceb_q3b: row count");
  if (t->movie_bound < 0 || t->person_bound < 0 || p->n_kind_codes < 0 || p->n_role_codes < 0 ||
      p->kind_mask_size < 0 || p->role_mask_size < 0 || p->company_map_size < 0 || p->title_len < 0 ||
      p->pcode_len < 0 || p->company_len < 0)
    return set_error(ctx, BO_ERR_INVALID, "ceb_q3b: negative size");
  const int32_t types[] = {p->title_type, p->pcode_type, p->company_type};
  for (int32_t ty : types)
    if (ty < kLikeAll || ty > kLikeGeneral) return set_error(ctx, BO_ERR_INVALID, "ceb_q3b: pattern kind");
  if (!col_ok(t->kt_id, t->n_kind_type) || !col_ok(t->kt_kind, t->n_kind_type) || !col_ok(t->rt_id, t->n_role_type) ||
      !col_ok(t->rt_role, t->n_role_type) || !col_ok(t->cn_id, t->n_company_name) ||
      !col_ok(t->cn_name, t->n_company_name) || !col_ok(t->mc_movie_id, t->n_movie_companies) ||
      !col_ok(t->mc_company_id, t->n_movie_companies) || !col_ok(t->mc_company_type_id, t->n_movie_companies) ||
      !col_ok(t->mk_movie_id, t->n_movie_keyword) || !col_ok(t->mk_keyword_id, t->n_movie_keyword) ||
      !col_ok(t->t_id, t->n_title) || !col_ok(t->t_title, t->n_title) || !col_ok(t->t_kind_id, t->n_title) ||
      !col_ok(t->ci_movie_id, t->n_cast_info) || !col_ok(t->ci_person_id, t->n_cast_info) ||
      !col_ok(t->ci_role_id, t->n_cast_info) || !col_ok(t->nm_id, t->n_name) || !col_ok(t->nm_name, t->n_name) ||
      !col_ok(t->nm_pcode, t->n_name))
    return set_error(ctx, BO_ERR_INVALID, "ceb_q3b: null column");
  const bo_ceb_dict* dicts[] = {&t->title_dict, &t->name_dict, &t->company_dict, &t->pcode_dict};
  for (const auto* d : dicts)
    if (d->n > 0 && (!d->offsets || !d->rank)) return set_error(ctx, BO_ERR_INVALID, "ceb_q3b: null dictionary");
  if ((p->n_kind_codes > 0 && !p->kind_allowed) || (p->n_role_codes > 0 && !p->role_allowed) ||
      (p->title_len > 0 && !p->title_pat) || (p->pcode_len > 0 && !p->pcode_pat) ||
      (p->company_len > 0 && !p->company_pat))
    return set_error(ctx, BO_ERR_INVALID, "ceb_q3b: null parameter array");
  const Pack pk{bits_for(t->name_dict.n), bits_for(t->company_dict.n)};
  if (bits_for(t->title_dict.n) + pk.nb + pk.cb > 64)
    return set_error(ctx, BO_ERR_UNSUPPORTED, "ceb_q3b: title, name and company codes exceed 64 bits");
  if (t->n_movie_companies == 0 || t->n_cast_info == 0 || t->n_movie_keyword == 0 || t->n_title == 0 ||
      t->n_name == 0 || t->movie_bound == 0 || t->person_bound == 0)
    return BO_OK;  // no movie can join: no rows
  const int64_t n_mc = t->n_movie_companies, n_ci = t->n_cast_info, MB = t->movie_bound, PB = t->person_bound;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += al256(std::max<size_t>(bytes, 1));
    return o;
  };
  const size_t o_meta = take(sizeof(Q3bMeta));
  const size_t o_kind = take((size_t)p->kind_mask_size), o_role = take((size_t)p->role_mask_size);
  const size_t o_inmc = take((size_t)MB), o_mk = take(4 * (size_t)MB), o_cand = take((size_t)PB);
  const size_t o_mcb = take(4 * (size_t)MB), o_mce = take(4 * (size_t)MB);
  const size_t zero_end = off;
  const size_t o_cname = take(4 * (size_t)p->company_map_size), o_title = take(4 * (size_t)MB);
  const size_t o_pname = take(4 * (size_t)PB);
  const size_t neg_end = off;  // these start at -1
  const size_t o_cm = take((size_t)t->company_dict.n), o_tm = take((size_t)t->title_dict.n);
  const size_t o_pm = take((size_t)t->pcode_dict.n);
  const int64_t nk = std::max(n_mc, n_ci);
  const size_t o_keys = take(8 * (size_t)nk), o_tkeys = take(8 * (size_t)nk);
  const size_t o_vals = take(4 * (size_t)nk), o_tvals = take(4 * (size_t)nk);
  const size_t o_flag = take(4 * (size_t)nk), o_pos = take(4 * ((size_t)nk + 1));
  const size_t o_mck = take(8 * (size_t)n_mc), o_mcs = take(4 * ((size_t)n_mc + 1));
  const size_t o_cik = take(8 * (size_t)n_ci), o_cis = take(4 * ((size_t)n_ci + 1));
  const size_t o_nruns = take(64);
  const size_t o_ka = take((size_t)p->n_kind_codes), o_ra = take((size_t)p->n_role_codes);
  const size_t o_tp = take((size_t)p->title_len), o_pp = take((size_t)p->pcode_len), o_cp = take((size_t)p->company_len);
  void* wsp = nullptr;
  int rc = region(ctx, "ceb_q3b_ws", off, &wsp);
  if (rc) return rc;
  char* ws = static_cast<char*>(wsp);
  auto* meta = reinterpret_cast<Q3bMeta*>(ws + o_meta);
  auto *kind_mask = reinterpret_cast<uint8_t*>(ws + o_kind), *role_mask = reinterpret_cast<uint8_t*>(ws + o_role);
  auto* in_mc = reinterpret_cast<uint8_t*>(ws + o_inmc);
  auto* mk = reinterpret_cast<unsigned int*>(ws + o_mk);
  auto* cand = reinterpret_cast<uint8_t*>(ws + o_cand);
  auto *mc_begin = reinterpret_cast<unsigned int*>(ws + o_mcb), *mc_end = reinterpret_cast<unsigned int*>(ws + o_mce);
  auto* cname = reinterpret_cast<int32_t*>(ws + o_cname);
  auto* title_of = reinterpret_cast<int32_t*>(ws + o_title);
  auto* pname = reinterpret_cast<int32_t*>(ws + o_pname);
  auto *cm = reinterpret_cast<uint8_t*>(ws + o_cm), *tm = reinterpret_cast<uint8_t*>(ws + o_tm);
  auto* pm = reinterpret_cast<uint8_t*>(ws + o_pm);
  auto *keys = reinterpret_cast<unsigned long long*>(ws + o_keys), *tkeys = reinterpret_cast<unsigned long long*>(ws + o_tkeys);
  auto *vals = reinterpret_cast<uint32_t*>(ws + o_vals), *tvals = reinterpret_cast<uint32_t*>(ws + o_tvals);
  auto *flag = reinterpret_cast<unsigned int*>(ws + o_flag), *pos = reinterpret_cast<unsigned int*>(ws + o_pos);
  auto* mck = reinterpret_cast<unsigned long long*>(ws + o_mck);
  auto* mcs = reinterpret_cast<unsigned int*>(ws + o_mcs);
  auto* cik = reinterpret_cast<unsigned long long*>(ws + o_cik);
  auto* cis = reinterpret_cast<unsigned int*>(ws + o_cis);
  auto* nruns = reinterpret_cast<unsigned int*>(ws + o_nruns);  // [0] mc runs, [1] cast runs
  auto *ka = reinterpret_cast<uint8_t*>(ws + o_ka), *ra = reinterpret_cast<uint8_t*>(ws + o_ra);
  auto *tp = reinterpret_cast<char*>(ws + o_tp), *pp = reinterpret_cast<char*>(ws + o_pp),
       *cp = reinterpret_cast<char*>(ws + o_cp);
  BO_CUDA(ctx, cudaMemsetAsync(ws, 0, zero_end, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(ws + zero_end, 0xff, neg_end - zero_end, ctx->stream));
  struct Copy {
    void* dst;
    const void* src;
    size_t n;
  } copies[] = {{ka, p->kind_allowed, (size_t)p->n_kind_codes}, {ra, p->role_allowed, (size_t)p->n_role_codes},
                {tp, p->title_pat, (size_t)p->title_len},      {pp, p->pcode_pat, (size_t)p->pcode_len},
                {cp, p->company_pat, (size_t)p->company_len}};
  for (const auto& c : copies)
    if (c.n > 0) BO_CUDA(ctx, cudaMemcpyAsync(c.dst, c.src, c.n, cudaMemcpyHostToDevice, ctx->stream));
  // masks and ILIKE
  const void* kd = reinterpret_cast<const void*>(&ceb_dim_mask_kernel);
  if (t->n_kind_type > 0) {
    ceb_dim_mask_kernel<<<q3b_grid(ctx, kd, t->n_kind_type), kCebBlock, 0, ctx->stream>>>(
        t->kt_id, t->kt_kind, t->n_kind_type, ka, p->n_kind_codes, p->kind_mask_size, kind_mask, &meta->any_kind);
    if ((rc = after_launch(ctx, "ceb_dim_mask_kernel"))) return rc;
  }
  if (t->n_role_type > 0) {
    ceb_dim_mask_kernel<<<q3b_grid(ctx, kd, t->n_role_type), kCebBlock, 0, ctx->stream>>>(
        t->rt_id, t->rt_role, t->n_role_type, ra, p->n_role_codes, p->role_mask_size, role_mask, &meta->any_role);
    if ((rc = after_launch(ctx, "ceb_dim_mask_kernel"))) return rc;
  }
  const void* kl = reinterpret_cast<const void*>(&ceb_like_dict_kernel);
  struct Like {
    const bo_ceb_dict* d;
    int32_t type;
    const char* pat;
    int32_t len;
    uint8_t* out;
  } likes[] = {{&t->company_dict, p->company_type, cp, p->company_len, cm},
               {&t->title_dict, p->title_type, tp, p->title_len, tm},
               {&t->pcode_dict, p->pcode_type, pp, p->pcode_len, pm}};
  for (const auto& l : likes) {
    if (l.d->n == 0) continue;
    ceb_like_dict_kernel<<<q3b_grid(ctx, kl, l.d->n), kCebBlock, 0, ctx->stream>>>(l.d->bytes, l.d->offsets, l.d->n,
                                                                                  l.type, l.pat, l.len, l.out);
    if ((rc = after_launch(ctx, "ceb_like_dict_kernel"))) return rc;
  }
  // companies -> (movie, company) runs
  if (t->n_company_name > 0) {
    const void* kc = reinterpret_cast<const void*>(&q3b_company_kernel);
    q3b_company_kernel<<<q3b_grid(ctx, kc, t->n_company_name), kCebBlock, 0, ctx->stream>>>(*t, cm,
                                                                                           p->company_map_size,
                                                                                           cname, meta);
    if ((rc = after_launch(ctx, "q3b_company_kernel"))) return rc;
  }
  const void* kmc = reinterpret_cast<const void*>(&q3b_mc_kernel);
  q3b_mc_kernel<<<q3b_grid(ctx, kmc, n_mc), kCebBlock, 0, ctx->stream>>>(*t, cname, p->company_map_size, keys, meta);
  if ((rc = after_launch(ctx, "q3b_mc_kernel"))) return rc;
  if ((rc = q3b_runs(ctx, keys, vals, tkeys, tvals, n_mc, &meta->n_mc, flag, pos, mck, mcs))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(nruns, pos + n_mc, 4, cudaMemcpyDeviceToDevice, ctx->stream));
  const void* kmr = reinterpret_cast<const void*>(&q3b_movie_range_kernel);
  q3b_movie_range_kernel<<<q3b_grid(ctx, kmr, n_mc), kCebBlock, 0, ctx->stream>>>(mck, nruns, mc_begin, mc_end, in_mc);
  if ((rc = after_launch(ctx, "q3b_movie_range_kernel"))) return rc;
  // keywords, titles
  const void* kmk = reinterpret_cast<const void*>(&q3b_mk_kernel);
  q3b_mk_kernel<<<q3b_grid(ctx, kmk, t->n_movie_keyword), kCebBlock, 0, ctx->stream>>>(*t, in_mc, mk);
  if ((rc = after_launch(ctx, "q3b_mk_kernel"))) return rc;
  const void* kt = reinterpret_cast<const void*>(&q3b_title_kernel);
  q3b_title_kernel<<<q3b_grid(ctx, kt, t->n_title), kCebBlock, 0, ctx->stream>>>(*t, in_mc, mk, kind_mask,
                                                                                p->kind_mask_size, tm, title_of);
  if ((rc = after_launch(ctx, "q3b_title_kernel"))) return rc;
  // cast -> (movie, person) runs; names
  const void* kci = reinterpret_cast<const void*>(&q3b_cast_kernel);
  q3b_cast_kernel<<<q3b_grid(ctx, kci, n_ci), kCebBlock, 0, ctx->stream>>>(*t, title_of, role_mask, p->role_mask_size,
                                                                          keys, cand, meta);
  if ((rc = after_launch(ctx, "q3b_cast_kernel"))) return rc;
  if ((rc = q3b_runs(ctx, keys, vals, tkeys, tvals, n_ci, &meta->n_ci, flag, pos, cik, cis))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(nruns + 1, pos + n_ci, 4, cudaMemcpyDeviceToDevice, ctx->stream));
  const void* knm = reinterpret_cast<const void*>(&q3b_name_kernel);
  q3b_name_kernel<<<q3b_grid(ctx, knm, t->n_name), kCebBlock, 0, ctx->stream>>>(*t, cand, pm, pname);
  if ((rc = after_launch(ctx, "q3b_name_kernel"))) return rc;
  const Runs ci{cik, cis, nruns + 1}, mc{mck, mcs, nruns};
  const void* kj0 = reinterpret_cast<const void*>(&q3b_join_kernel<false>);
  const int gj = q3b_grid(ctx, kj0, n_ci);
  q3b_join_kernel<false><<<gj, kCebBlock, 0, ctx->stream>>>(ci, mc, mc_begin, mc_end, mk, title_of, pname, cname, PB,
                                                            pk, nullptr, nullptr, 0, meta);
  if ((rc = after_launch(ctx, "q3b_join_kernel"))) return rc;
  // One host round trip sizes the group table.
  Q3bMeta m{};
  BO_CUDA(ctx, cudaMemcpyAsync(&m, meta, sizeof(m), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (!m.any_kind || !m.any_role || !m.any_comp || m.expansions == 0) return BO_OK;
  unsigned long long slots = 1024;
  while (slots < 2 * m.expansions) slots <<= 1;
  const size_t hb = al256(8 * slots);
  const size_t outb = al256(8 * (size_t)m.expansions);
  const size_t rowb = al256(sizeof(bo_ceb_q3b_row) * (size_t)m.expansions);
  void* hp = nullptr;
  if ((rc = region(ctx, "ceb_q3b_groups", 2 * hb + 4 * outb + 2 * al256(4 * (size_t)m.expansions) + rowb, &hp)))
    return rc;
  char* hbp = static_cast<char*>(hp);
  auto* hkeys = reinterpret_cast<unsigned long long*>(hbp);
  auto* hcount = reinterpret_cast<unsigned long long*>(hbp + hb);
  auto* okey = reinterpret_cast<unsigned long long*>(hbp + 2 * hb);
  auto* ocount = reinterpret_cast<unsigned long long*>(hbp + 2 * hb + outb);
  auto* sk = reinterpret_cast<unsigned long long*>(hbp + 2 * hb + 2 * outb);
  auto* tsk = reinterpret_cast<unsigned long long*>(hbp + 2 * hb + 3 * outb);
  auto* idx = reinterpret_cast<uint32_t*>(hbp + 2 * hb + 4 * outb);
  auto* tidx = reinterpret_cast<uint32_t*>(hbp + 2 * hb + 4 * outb + al256(4 * (size_t)m.expansions));
  auto* rows_dev = reinterpret_cast<bo_ceb_q3b_row*>(hbp + 2 * hb + 4 * outb + 2 * al256(4 * (size_t)m.expansions));
  BO_CUDA(ctx, cudaMemsetAsync(hkeys, 0xff, 8 * slots, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(hcount, 0, 8 * slots, ctx->stream));
  q3b_join_kernel<true><<<gj, kCebBlock, 0, ctx->stream>>>(ci, mc, mc_begin, mc_end, mk, title_of, pname, cname, PB, pk,
                                                           hkeys, hcount, slots - 1, meta);
  if ((rc = after_launch(ctx, "q3b_join_kernel"))) return rc;
  const void* ke = reinterpret_cast<const void*>(&q3b_emit_kernel);
  q3b_emit_kernel<<<q3b_grid(ctx, ke, (int64_t)slots), kCebBlock, 0, ctx->stream>>>(hkeys, hcount, slots, okey, ocount,
                                                                                   meta);
  if ((rc = after_launch(ctx, "q3b_emit_kernel"))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(&m, meta, sizeof(m), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (m.bad) return set_error(ctx, BO_ERR_OVERFLOW, "ceb_q3b: group table full");
  const int64_t n_rows = (int64_t)m.n_rows;
  *n_rows_out = n_rows;
  if (n_rows > max_rows)
    return set_error(ctx, BO_ERR_OVERFLOW, "ceb_q3b: %lld groups, room for %lld", (long long)n_rows,
                     (long long)max_rows);
  if (n_rows == 0) return BO_OK;
  // ORDER BY count desc, title, name, company (two stable radix sorts).
  const void* krk = reinterpret_cast<const void*>(&q3b_rank_key_kernel);
  q3b_rank_key_kernel<<<q3b_grid(ctx, krk, n_rows), kCebBlock, 0, ctx->stream>>>(
      okey, n_rows, pk, t->title_dict.rank, t->name_dict.rank, t->company_dict.rank, sk, idx);
  if ((rc = after_launch(ctx, "q3b_rank_key_kernel"))) return rc;
  if ((rc = radix_sort_pairs(ctx, sk, idx, tsk, tidx, n_rows, 0, 64, nullptr))) return rc;
  const void* kck = reinterpret_cast<const void*>(&q3b_count_key_kernel);
  q3b_count_key_kernel<<<q3b_grid(ctx, kck, n_rows), kCebBlock, 0, ctx->stream>>>(ocount, idx, n_rows, sk);
  if ((rc = after_launch(ctx, "q3b_count_key_kernel"))) return rc;
  if ((rc = radix_sort_pairs(ctx, sk, idx, tsk, tidx, n_rows, 0, 64, nullptr))) return rc;
  const void* kro = reinterpret_cast<const void*>(&q3b_rows_kernel);
  q3b_rows_kernel<<<q3b_grid(ctx, kro, n_rows), kCebBlock, 0, ctx->stream>>>(okey, ocount, idx, n_rows, pk, rows_dev);
  if ((rc = after_launch(ctx, "q3b_rows_kernel"))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(rows_out, rows_dev, sizeof(bo_ceb_q3b_row) * (size_t)n_rows, cudaMemcpyDeviceToHost,
                               ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // synchronises the stream
  return device_error_status(ctx, bits, "ceb_q3b");
}
