// CEB query 1a: run_q1a of bespoke_ceb/query_q1a.cpp:155-655.
//
// The reference builds byte masks of the allowed kind / role / person ids
// from the dimension tables, scans title for the qualifying movies, counts
// per movie the movie_info rows matching (ID1, INFO1) and (ID2, INFO2), then
// the cast_info rows of the movies with both counts and an allowed role and
// person, and sums cast * count1 * count2 over the qualifying title rows
// (the factorised count of the join, :605-624).  Here every step is a pass
// over device columns in the reference's own layout (int32 values plus an
// optional null byte per row):
//   ceb_dim_mask_kernel   id mask of a dimension table (one launch per table);
//   ceb_title_kernel      qualifying title rows -> a list of movie ids
//                         (warp-aggregated reservations) and the largest id;
//   ceb_info_kernel       dense per-movie counts of the two info predicates;
//   ceb_both_kernel       the movies with both counts;
//   ceb_cast_kernel       dense per-movie cast counts, lanes of a warp with
//                         the same movie combined (match_any) before the
//                         atomic, for the skewed movie ids;
//   ceb_sum_kernel        the factorised sum over the title list.
#include <algorithm>

#include "ceb.cuh"
#include "context.cuh"

namespace bo {
namespace {

struct CebMeta {
  unsigned int n_list;
  int max_movie;
  unsigned long long total;
};

__global__ void __launch_bounds__(kCebBlock) ceb_title_kernel(bo_ceb_q1a_tables t, int32_t year1, int32_t year2,
                                                              const uint8_t* __restrict__ kind_mask,
                                                              int32_t kind_mask_size, int32_t* __restrict__ list,
                                                              CebMeta* __restrict__ meta) {
  int best = -1;
  const int64_t n = t.n_title;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  const int64_t n_warp = (n + 31) & ~int64_t(31);  // whole warps iterate together (warp_append)
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < n_warp; r += stride) {
    bool take = false;
    int32_t movie = 0;
    if (r < n && !ceb_null(t.t_id, r) && !ceb_null(t.t_year, r) && !ceb_null(t.t_kind_id, r)) {
      movie = t.t_id.values[r];
      const int32_t year = t.t_year.values[r], kind = t.t_kind_id.values[r];
      take = movie >= 0 && year <= year1 && year >= year2 && kind >= 0 && kind < kind_mask_size && kind_mask[kind];
    }
    warp_append<int32_t>(take, movie, list, &meta->n_list);
    if (take) best = max(best, movie);
  }
  for (int o = 16; o; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0 && best >= 0) atomicMax(&meta->max_movie, best);
}

__global__ void __launch_bounds__(kCebBlock) ceb_info_kernel(bo_ceb_q1a_tables t,
                                                             const uint8_t* __restrict__ type_filter,
                                                             int32_t type_size, const uint8_t* __restrict__ match,
                                                             int32_t n_codes, const CebMeta* __restrict__ meta,
                                                             unsigned int* __restrict__ c1,
                                                             unsigned int* __restrict__ c2) {
  const int max_movie = meta->max_movie;
  if (max_movie < 0) return;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < t.n_movie_info; r += stride) {
    if (ceb_null(t.mi_info_type_id, r)) continue;
    const uint32_t type = (uint32_t)t.mi_info_type_id.values[r];
    if (type >= (uint32_t)type_size) continue;
    const uint32_t f = type_filter[type];
    if (!f || ceb_null(t.mi_info, r)) continue;
    const int32_t code = t.mi_info.values[r];
    const uint32_t m = (code >= 0 && code < n_codes) ? match[code] : 0u;
    const uint32_t hit = f & m;
    if (!hit || ceb_null(t.mi_movie_id, r)) continue;
    const int32_t movie = t.mi_movie_id.values[r];
    if (movie < 0 || movie > max_movie) continue;
    if (hit & 1u) atomicAdd(c1 + movie, 1u);
    if (hit & 2u) atomicAdd(c2 + movie, 1u);
  }
}

__global__ void __launch_bounds__(kCebBlock) ceb_both_kernel(const int32_t* __restrict__ list,
                                                             const CebMeta* __restrict__ meta,
                                                             const unsigned int* __restrict__ c1,
                                                             const unsigned int* __restrict__ c2,
                                                             uint8_t* __restrict__ both) {
  const int64_t n = meta->n_list;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t i = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; i < n; i += stride) {
    const int32_t m = list[i];
    if (c1[m] && c2[m]) both[m] = 1;
  }
}

__global__ void __launch_bounds__(kCebBlock) ceb_cast_kernel(bo_ceb_q1a_tables t, const uint8_t* __restrict__ both,
                                                             const uint8_t* __restrict__ role_mask,
                                                             int32_t role_mask_size,
                                                             const uint8_t* __restrict__ person_mask,
                                                             int32_t person_mask_size,
                                                             const CebMeta* __restrict__ meta,
                                                             unsigned int* __restrict__ cast) {
  const int max_movie = meta->max_movie;
  if (max_movie < 0) return;
  const int64_t n = t.n_cast_info;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  const int64_t n_warp = (n + 31) & ~int64_t(31);
  const int lane = threadIdx.x & 31;
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < n_warp; r += stride) {
    int32_t movie = -1;
    if (r < n && !ceb_null(t.ci_movie_id, r)) {
      const int32_t m = t.ci_movie_id.values[r];
      if (m >= 0 && m <= max_movie && both[m] && !ceb_null(t.ci_role_id, r) && !ceb_null(t.ci_person_id, r)) {
        const int32_t role = t.ci_role_id.values[r], person = t.ci_person_id.values[r];
        if (role >= 0 && role < role_mask_size && role_mask[role] && person >= 0 && person < person_mask_size &&
            person_mask[person])
          movie = m;
      }
    }
    // Lanes counting the same movie add once (skewed movie ids).
    const unsigned int peers = __match_any_sync(0xffffffffu, movie);
    if (movie >= 0 && lane == __ffs(peers) - 1) atomicAdd(cast + movie, (unsigned int)__popc(peers));
  }
}

__global__ void __launch_bounds__(kCebBlock) ceb_sum_kernel(const int32_t* __restrict__ list,
                                                            CebMeta* __restrict__ meta,
                                                            const unsigned int* __restrict__ c1,
                                                            const unsigned int* __restrict__ c2,
                                                            const unsigned int* __restrict__ cast) {
  const int64_t n = meta->n_list;
  unsigned long long s = 0;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t i = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; i < n; i += stride) {
    const int32_t m = list[i];
    s += (unsigned long long)cast[m] * c1[m] * c2[m];
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ unsigned long long part[kCebBlock / 32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long b = 0;
    for (int w = 0; w < kCebBlock / 32; ++w) b += part[w];
    if (b) atomicAdd(&meta->total, b);
  }
}

int ceb_grid(bo_ctx* ctx, const void* k, int64_t threads) {
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(k, kCebBlock, 0);
  return (int)std::max<int64_t>(1, std::min<int64_t>((threads + kCebBlock - 1) / kCebBlock, resident));
}

size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

bool col_ok(const bo_ceb_col& c, int64_t n) { return n == 0 || c.values; }

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_ceb_q1a(bo_ctx* ctx, const bo_ceb_q1a_tables* t, const bo_ceb_q1a_params* p, int64_t* count_out) {
  BO_CHECK_CTX(ctx);
  if (!t || !p || !count_out) return set_error(ctx, BO_ERR_INVALID, "ceb_q1a: null argument");
  *count_out = 0;
  const int64_t ns[] = {t->n_title, t->n_movie_info, t->n_cast_info, t->n_kind_type, t->n_role_type, t->n_name};
  for (int64_t n : ns)
    if (n < 0) return set_error(ctx, BO_ERR_INVALID, "ceb_q1a: negative row count");
  const int32_t sizes[] = {p->info_type_size, p->n_info_codes, p->n_kind_codes, p->n_role_codes, p->n_gender_codes,
                           p->kind_mask_size, p->role_mask_size, p->person_mask_size};
  for (int32_t v : sizes)
    if (v < 0) return set_error(ctx, BO_ERR_INVALID, "ceb_q1a: negative size");
  if (!col_ok(t->t_id, t->n_title) || !col_ok(t->t_kind_id, t->n_title) || !col_ok(t->t_year, t->n_title) ||
      !col_ok(t->mi_movie_id, t->n_movie_info) || !col_ok(t->mi_info_type_id, t->n_movie_info) ||
      !col_ok(t->mi_info, t->n_movie_info) || !col_ok(t->ci_movie_id, t->n_cast_info) ||
      !col_ok(t->ci_person_id, t->n_cast_info) || !col_ok(t->ci_role_id, t->n_cast_info) ||
      !col_ok(t->kt_id, t->n_kind_type) || !col_ok(t->kt_kind, t->n_kind_type) || !col_ok(t->rt_id, t->n_role_type) ||
      !col_ok(t->rt_role, t->n_role_type) || !col_ok(t->nm_id, t->n_name) || !col_ok(t->nm_gender, t->n_name))
    return set_error(ctx, BO_ERR_INVALID, "ceb_q1a: null column");
  if ((p->info_type_size > 0 && !p->info_type_filter) || (p->n_info_codes > 0 && !p->info_match) ||
      (p->n_kind_codes > 0 && !p->kind_allowed) || (p->n_role_codes > 0 && !p->role_allowed) ||
      (p->n_gender_codes > 0 && !p->gender_allowed))
    return set_error(ctx, BO_ERR_INVALID, "ceb_q1a: null parameter array");
  if (t->n_title == 0 || t->max_title_id < 0) return BO_OK;  // no title row: the count is 0 (:273-275)
  if (t->n_title > 0x7fffffffll) return set_error(ctx, BO_ERR_INVALID, "ceb_q1a: title above 2^31 rows");
  const size_t n_movies = (size_t)t->max_title_id + 1;
  // Workspace: meta | title list | c1 | c2 | cast | both | masks | small host arrays.
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += al256(std::max<size_t>(bytes, 1));
    return o;
  };
  const size_t o_meta = take(sizeof(CebMeta));
  const size_t o_list = take(4 * (size_t)t->n_title);
  const size_t o_c1 = take(4 * n_movies), o_c2 = take(4 * n_movies), o_cast = take(4 * n_movies);
  const size_t o_both = take(n_movies);
  const size_t o_kind = take((size_t)p->kind_mask_size), o_role = take((size_t)p->role_mask_size);
  const size_t o_person = take((size_t)p->person_mask_size);
  const size_t zero_end = off;  // everything up to here starts at zero
  const size_t o_tf = take((size_t)p->info_type_size), o_match = take((size_t)p->n_info_codes);
  const size_t o_ka = take((size_t)p->n_kind_codes), o_ra = take((size_t)p->n_role_codes);
  const size_t o_ga = take((size_t)p->n_gender_codes);
  void* wsp = nullptr;
  int rc = region(ctx, "ceb_q1a_ws", off, &wsp);
  if (rc) return rc;
  char* ws = static_cast<char*>(wsp);
  auto* meta = reinterpret_cast<CebMeta*>(ws + o_meta);
  auto* list = reinterpret_cast<int32_t*>(ws + o_list);
  auto* c1 = reinterpret_cast<unsigned int*>(ws + o_c1);
  auto* c2 = reinterpret_cast<unsigned int*>(ws + o_c2);
  auto* cast = reinterpret_cast<unsigned int*>(ws + o_cast);
  auto* both = reinterpret_cast<uint8_t*>(ws + o_both);
  auto *kind_mask = reinterpret_cast<uint8_t*>(ws + o_kind), *role_mask = reinterpret_cast<uint8_t*>(ws + o_role);
  auto* person_mask = reinterpret_cast<uint8_t*>(ws + o_person);
  auto *tf = reinterpret_cast<uint8_t*>(ws + o_tf), *match = reinterpret_cast<uint8_t*>(ws + o_match);
  auto *ka = reinterpret_cast<uint8_t*>(ws + o_ka), *ra = reinterpret_cast<uint8_t*>(ws + o_ra);
  auto* ga = reinterpret_cast<uint8_t*>(ws + o_ga);
  BO_CUDA(ctx, cudaMemsetAsync(ws, 0, zero_end, ctx->stream));
  {
    const CebMeta m0{0u, -1, 0ull};
    BO_CUDA(ctx, cudaMemcpyAsync(meta, &m0, sizeof(m0), cudaMemcpyHostToDevice, ctx->stream));
  }
  struct Copy {
    void* dst;
    const void* src;
    int32_t n;
  } copies[] = {{tf, p->info_type_filter, p->info_type_size},
                {match, p->info_match, p->n_info_codes},
                {ka, p->kind_allowed, p->n_kind_codes},
                {ra, p->role_allowed, p->n_role_codes},
                {ga, p->gender_allowed, p->n_gender_codes}};
  for (const auto& c : copies)
    if (c.n > 0) BO_CUDA(ctx, cudaMemcpyAsync(c.dst, c.src, (size_t)c.n, cudaMemcpyHostToDevice, ctx->stream));
  const void* kd = reinterpret_cast<const void*>(&ceb_dim_mask_kernel);
  struct Dim {
    bo_ceb_col id, code;
    int64_t n;
    const uint8_t* allowed;
    int32_t n_codes, size;
    uint8_t* mask;
  } dims[] = {{t->kt_id, t->kt_kind, t->n_kind_type, ka, p->n_kind_codes, p->kind_mask_size, kind_mask},
              {t->rt_id, t->rt_role, t->n_role_type, ra, p->n_role_codes, p->role_mask_size, role_mask},
              {t->nm_id, t->nm_gender, t->n_name, ga, p->n_gender_codes, p->person_mask_size, person_mask}};
  for (const auto& d : dims) {
    if (d.n == 0 || d.size == 0) continue;
    ceb_dim_mask_kernel<<<ceb_grid(ctx, kd, d.n), kCebBlock, 0, ctx->stream>>>(d.id, d.code, d.n, d.allowed,
                                                                             d.n_codes, d.size, d.mask, nullptr);
    if ((rc = after_launch(ctx, "ceb_dim_mask_kernel"))) return rc;
  }
  const void* kt = reinterpret_cast<const void*>(&ceb_title_kernel);
  ceb_title_kernel<<<ceb_grid(ctx, kt, t->n_title), kCebBlock, 0, ctx->stream>>>(
      *t, p->year1, p->year2, kind_mask, p->kind_mask_size, list, meta);
  if ((rc = after_launch(ctx, "ceb_title_kernel"))) return rc;
  if (t->n_movie_info > 0) {
    const void* ki = reinterpret_cast<const void*>(&ceb_info_kernel);
    ceb_info_kernel<<<ceb_grid(ctx, ki, t->n_movie_info), kCebBlock, 0, ctx->stream>>>(
        *t, tf, p->info_type_size, match, p->n_info_codes, meta, c1, c2);
    if ((rc = after_launch(ctx, "ceb_info_kernel"))) return rc;
  }
  const void* kb = reinterpret_cast<const void*>(&ceb_both_kernel);
  ceb_both_kernel<<<ceb_grid(ctx, kb, t->n_title), kCebBlock, 0, ctx->stream>>>(list, meta, c1, c2, both);
  if ((rc = after_launch(ctx, "ceb_both_kernel"))) return rc;
  if (t->n_cast_info > 0) {
    const void* kc = reinterpret_cast<const void*>(&ceb_cast_kernel);
    ceb_cast_kernel<<<ceb_grid(ctx, kc, t->n_cast_info), kCebBlock, 0, ctx->stream>>>(
        *t, both, role_mask, p->role_mask_size, person_mask, p->person_mask_size, meta, cast);
    if ((rc = after_launch(ctx, "ceb_cast_kernel"))) return rc;
  }
  const void* ks = reinterpret_cast<const void*>(&ceb_sum_kernel);
  ceb_sum_kernel<<<ceb_grid(ctx, ks, t->n_title), kCebBlock, 0, ctx->stream>>>(list, meta, c1, c2, cast);
  if ((rc = after_launch(ctx, "ceb_sum_kernel"))) return rc;
  CebMeta out{};
  BO_CUDA(ctx, cudaMemcpyAsync(&out, meta, sizeof(out), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *count_out = (int64_t)out.total;
  return BO_OK;
}
