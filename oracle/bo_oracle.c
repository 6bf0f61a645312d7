/*
 * ORACLE -- test infrastructure, not part of the product.
 *
 * Plain-C restatement of the reference pipelines this engine replaces.  Only the
 * tests, the smoke check and bench.py's CPU-baseline leg load it, and only as
 * the checker; the GPU engine never calls, links or falls back to it.
 *
 * Each function cites the reference loop it restates (paths relative to the
 * DataManagementLab/BespokeOLAP_Artifacts tree).  All arithmetic is exact
 * integer arithmetic with __int128 totals, as in the reference.
 *
 * Parity pinning: the reference ships no golden vectors or tests.  The
 * restatement is pinned by running the reference's own compiled pipelines
 * (oracle/ref_harness.cpp, built from the reference sources into oracle/_ref/)
 * on the same seeded inputs; see tests/test_oracle_pin.py.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef __int128 i128;

typedef struct o_i128 {
  uint64_t lo;
  int64_t hi;
} o_i128;

/* Same field order as bo_q1_agg (include/bespoke_gpu.h). */
typedef struct o_q1_agg {
  int64_t count;
  int64_t sum_qty;
  int64_t sum_base_price;
  int64_t sum_disc;
  int64_t sum_disc_price;
  int64_t sum_disc_price_exact;
  o_i128 sum_charge;
  o_i128 sum_charge_exact;
} o_q1_agg;

static o_i128 put128(i128 v) {
  o_i128 r;
  r.lo = (uint64_t)v;
  r.hi = (int64_t)(v >> 64);
  return r;
}

typedef struct q1_acc {
  i128 count, qty, price, disc, dp, dpe, ch, che;
} q1_acc;

static void q1_emit(const q1_acc* a, o_q1_agg* out) {
  out->count = (int64_t)a->count;
  out->sum_qty = (int64_t)a->qty;
  out->sum_base_price = (int64_t)a->price;
  out->sum_disc = (int64_t)a->disc;
  out->sum_disc_price = (int64_t)a->dp;
  out->sum_disc_price_exact = (int64_t)a->dpe;
  out->sum_charge = put128(a->ch);
  out->sum_charge_exact = put128(a->che);
}

/* Q1 over the declared wide layout.  Restates run_q1's per-row update
 * (bespoke_tpch/query_q1.cpp:175-194) with the builder's derived column
 * discounted_price = trunc(price*(100-disc)/100) (builder_impl.cpp:527-531)
 * computed inline, plus the exact forms price*(100-disc)[*(100+tax)].
 * Returns 0, or -6 if a passing row has a group code outside the domain. */
int oracle_q1_fact(const int32_t* ship, const int64_t* qty, const int64_t* price, const int64_t* disc,
                   const int64_t* tax, const uint8_t* fa, const uint8_t* fb, int64_t n, int32_t cutoff,
                   int32_t n_fa, int32_t n_fb, o_q1_agg* out) {
  q1_acc acc[8];
  memset(acc, 0, sizeof(acc));
  int rc = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (ship[i] > cutoff) continue;
    if (fa[i] >= n_fa || fb[i] >= n_fb) {
      rc = -6;
      continue;
    }
    q1_acc* a = &acc[fa[i] * n_fb + fb[i]];
    const int64_t p1 = price[i] * (100 - disc[i]);
    const int64_t dp = p1 / 100; /* C++ truncation, as the builder does */
    const int64_t tm = 100 + tax[i];
    a->count += 1;
    a->qty += qty[i];
    a->price += price[i];
    a->disc += disc[i];
    a->dp += dp;
    a->dpe += p1;
    a->ch += (i128)(dp * tm);
    a->che += (i128)p1 * tm;
  }
  for (int g = 0; g < n_fa * n_fb; ++g) q1_emit(&acc[g], &out[g]);
  return rc;
}

/* Q1 over the reference storage-plan layout: exactly run_q1's scan
 * (bespoke_tpch/query_q1.cpp:125-230) -- filter shipdate <= cutoff, group by
 * the returnflag_linestatus code, sums of quantity, extendedprice,
 * discounted_price, discounted_price*(100+tax) (__int128), discount, count. */
int oracle_q1_lineitem(const int16_t* shipdate, const uint8_t* code, const int32_t* extendedprice,
                       const int32_t* discounted_price, const uint8_t* discount, const uint8_t* tax,
                       const int16_t* quantity, int64_t n, int16_t cutoff, int32_t n_groups, o_q1_agg* out) {
  q1_acc acc[8];
  memset(acc, 0, sizeof(acc));
  int rc = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (shipdate[i] > cutoff) continue;
    if (code[i] >= n_groups) {
      rc = -6;
      continue;
    }
    q1_acc* a = &acc[code[i]];
    const int32_t tm = 100 + (int32_t)tax[i];
    const int64_t p1 = (int64_t)extendedprice[i] * (100 - (int32_t)discount[i]);
    a->count += 1;
    a->qty += quantity[i];
    a->price += extendedprice[i];
    a->disc += discount[i];
    a->dp += discounted_price[i];
    a->dpe += p1;
    a->ch += (i128)((int64_t)discounted_price[i] * tm);
    a->che += (i128)p1 * tm;
  }
  for (int g = 0; g < n_groups; ++g) q1_emit(&acc[g], &out[g]);
  return rc;
}

/* run_q1's finalisation of one group (bespoke_tpch/query_q1.cpp:245-257):
 * integer totals to the doubles of Q1ResultRow, same expressions, same order. */
void oracle_q1_finalize(const o_q1_agg* a, double out[7]) {
  const double count = (double)a->count;
  const i128 ch = (i128)(((unsigned __int128)(uint64_t)a->sum_charge.hi << 64) | a->sum_charge.lo);
  out[0] = (double)a->sum_qty / 100;                /* sum_qty */
  out[1] = (double)a->sum_base_price / 100;         /* sum_base_price */
  out[2] = (double)a->sum_disc_price / 100;         /* sum_disc_price */
  out[3] = (double)ch / ((double)100 * 100);        /* sum_charge */
  out[4] = out[0] / count;                          /* avg_qty */
  out[5] = out[1] / count;                          /* avg_price */
  out[6] = (double)a->sum_disc / 100 / count;       /* avg_disc */
}

/* Q6 over the storage-plan layout: run_q6's unsharded scan
 * (bespoke_tpch/query_q6.cpp:197-222).  The sharded path (:224-379) visits the
 * same qualifying rows, so the total is the same. */
int oracle_q6_lineitem(const int16_t* shipdate, const int32_t* extendedprice, const uint8_t* discount,
                       const int16_t* quantity, int64_t n, int16_t start, int16_t end, int32_t dmin,
                       int32_t dmax, int32_t qlimit, int64_t* revenue, int64_t* count) {
  const uint32_t span = (uint32_t)((int32_t)end - (int32_t)start);
  const uint32_t dspan = (uint32_t)(dmax - dmin);
  i128 rev = 0;
  int64_t c = 0;
  for (int64_t i = 0; i < n; ++i) {
    if ((uint32_t)((int32_t)shipdate[i] - start) >= span) continue;
    if ((uint32_t)((int32_t)discount[i] - dmin) > dspan) continue;
    if ((int32_t)quantity[i] >= qlimit) continue;
    rev += (int64_t)extendedprice[i] * (int64_t)discount[i];
    c += 1;
  }
  *revenue = (int64_t)rev;
  *count = c;
  return 0;
}

/* ------------------------------------------------------------- hash join -- */
typedef struct kv_table {
  int32_t* keys;
  int64_t* vals;
  uint8_t* used;
  uint64_t mask;
} kv_table;

static uint32_t mix32(uint32_t k) {
  k ^= k >> 16;
  k *= 0x85ebca6bu;
  k ^= k >> 13;
  k *= 0xc2b2ae35u;
  k ^= k >> 16;
  return k;
}

static int kv_init(kv_table* t, int64_t n) {
  uint64_t cap = 16;
  while (cap < (uint64_t)n * 2) cap <<= 1;
  t->keys = (int32_t*)calloc(cap, sizeof(int32_t));
  t->vals = (int64_t*)calloc(cap, sizeof(int64_t));
  t->used = (uint8_t*)calloc(cap, 1);
  t->mask = cap - 1;
  return (t->keys && t->vals && t->used) ? 0 : -2;
}

static void kv_free(kv_table* t) {
  free(t->keys);
  free(t->vals);
  free(t->used);
}

static int64_t* kv_slot(kv_table* t, int32_t key, int create) {
  uint64_t h = mix32((uint32_t)key) & t->mask;
  while (t->used[h]) {
    if (t->keys[h] == key) return &t->vals[h];
    h = (h + 1) & t->mask;
  }
  if (!create) return 0;
  t->used[h] = 1;
  t->keys[h] = key;
  t->vals[h] = 0;
  return &t->vals[h];
}

/* Filtered inner join + scalar aggregate (the filtered-join shape of run_q3,
 * bespoke_tpch/query_q3.cpp:182-260).  Build rows qualify when date < date_lt
 * and segment == seg_eq; every probe row whose fk equals a qualifying build key
 * contributes once per matching build row.  Outputs: qualifying build rows,
 * match count, sum price*(100-disc) (exact) and sum trunc(price*(100-disc)/100)
 * (the reference's discounted_price, builder_impl.cpp:527-531). */
int oracle_join_agg(const int32_t* bkey, const int32_t* bdate, const uint8_t* bseg, int64_t nb,
                    int32_t date_lt, int32_t seg_eq, const int32_t* pfk, const int64_t* pprice,
                    const int64_t* pdisc, int64_t np, int64_t* build_count, int64_t* match_count,
                    o_i128* sum_exact, o_i128* sum_trunc) {
  int64_t nq = 0;
  for (int64_t i = 0; i < nb; ++i) nq += (bdate[i] < date_lt && bseg[i] == seg_eq);
  kv_table t;
  if (kv_init(&t, nq)) {
    kv_free(&t);
    return -2;
  }
  for (int64_t i = 0; i < nb; ++i)
    if (bdate[i] < date_lt && bseg[i] == seg_eq) *kv_slot(&t, bkey[i], 1) += 1;
  i128 se = 0, st = 0;
  int64_t m = 0;
  for (int64_t i = 0; i < np; ++i) {
    const int64_t* mult = kv_slot(&t, pfk[i], 0);
    if (!mult) continue;
    const int64_t p1 = pprice[i] * (100 - pdisc[i]);
    m += *mult;
    se += (i128)p1 * *mult;
    st += (i128)(p1 / 100) * *mult;
  }
  kv_free(&t);
  *build_count = nq;
  *match_count = m;
  *sum_exact = put128(se);
  *sum_trunc = put128(st);
  return 0;
}

/* ---------------------------------------- group-by + radix sort + top-k -- */
typedef struct grp_entry {
  int32_t key;
  int32_t min_year;
  int64_t count;
} grp_entry;

/* Stable LSD counting sort with 16-bit digits, ordered by (count desc, key
 * asc): two passes over the key, then four over ~(uint64)count -- the scheme
 * of radix_sort_groups (bespoke_tpch/query_q10.cpp:318-372), where later passes
 * on the primary key keep the earlier key order among ties. */
static int radix_sort_groups(grp_entry* g, int64_t n) {
  if (n < 2) return 0;
  grp_entry* tmp = (grp_entry*)malloc(sizeof(grp_entry) * (size_t)n);
  uint32_t* counts = (uint32_t*)malloc(sizeof(uint32_t) * 65536);
  if (!tmp || !counts) {
    free(tmp);
    free(counts);
    return -2;
  }
  grp_entry* src = g;
  grp_entry* dst = tmp;
  for (int pass = 0; pass < 6; ++pass) {
    memset(counts, 0, sizeof(uint32_t) * 65536);
    for (int64_t i = 0; i < n; ++i) {
      const uint64_t k = pass < 2 ? (uint64_t)(uint32_t)src[i].key : ~(uint64_t)src[i].count;
      const int shift = pass < 2 ? 16 * pass : 16 * (pass - 2);
      counts[(k >> shift) & 0xffffu] += 1;
    }
    uint32_t sum = 0;
    for (int d = 0; d < 65536; ++d) {
      const uint32_t c = counts[d];
      counts[d] = sum;
      sum += c;
    }
    for (int64_t i = 0; i < n; ++i) {
      const uint64_t k = pass < 2 ? (uint64_t)(uint32_t)src[i].key : ~(uint64_t)src[i].count;
      const int shift = pass < 2 ? 16 * pass : 16 * (pass - 2);
      dst[counts[(k >> shift) & 0xffffu]++] = src[i];
    }
    grp_entry* t = src;
    src = dst;
    dst = t;
  }
  /* six passes: the result is back in g */
  free(tmp);
  free(counts);
  return 0;
}

/* Skewed three-way join + high-cardinality group-by + top-k.
 * Restates the dense-mask / dense-count pattern of run_q1a
 * (bespoke_ceb/query_q1a.cpp: dimension masks before :156, the cast_info scan
 * :503-601 with its bounds checks) with a min aggregate as in run_q10a
 * (bespoke_ceb/query_q10a.cpp:843-856) and the ordering of radix_sort_groups.
 *   C qualifies when its category is in cat_set and year_lo <= year <= year_hi;
 *   B row (a, c) joins when 0 <= c < nc, C[c] qualifies and a is an id of A;
 *   group by a: count, min(C.year); order by count desc, a asc; first k.
 * Returns the number of groups; writes min(k, groups) rows. */
int64_t oracle_groupby_topk(const int32_t* a_ids, int64_t na, const int32_t* b_a, const int32_t* b_c, int64_t nb,
                            const uint16_t* c_cat, const int32_t* c_year, int64_t nc, const uint16_t* cat_set,
                            int32_t n_cat, int32_t year_lo, int32_t year_hi, int32_t k, int32_t* out_key,
                            int64_t* out_count, int32_t* out_min_year, int64_t* joined_rows) {
  int32_t max_a = -1;
  for (int64_t i = 0; i < na; ++i)
    if (a_ids[i] > max_a) max_a = a_ids[i];
  const int64_t a_cap = (int64_t)max_a + 1;
  uint8_t* a_mask = (uint8_t*)calloc((size_t)(a_cap > 0 ? a_cap : 1), 1);
  uint8_t cat_mask[65536];
  memset(cat_mask, 0, sizeof(cat_mask));
  for (int i = 0; i < n_cat; ++i) cat_mask[cat_set[i]] = 1;
  uint8_t* c_ok = (uint8_t*)malloc((size_t)(nc > 0 ? nc : 1));
  int64_t* cnt = (int64_t*)calloc((size_t)(a_cap > 0 ? a_cap : 1), sizeof(int64_t));
  int32_t* mny = (int32_t*)malloc(sizeof(int32_t) * (size_t)(a_cap > 0 ? a_cap : 1));
  if (!a_mask || !c_ok || !cnt || !mny) {
    free(a_mask);
    free(c_ok);
    free(cnt);
    free(mny);
    return -2;
  }
  for (int64_t i = 0; i < na; ++i)
    if (a_ids[i] >= 0) a_mask[a_ids[i]] = 1;
  for (int64_t c = 0; c < nc; ++c)
    c_ok[c] = cat_mask[c_cat[c]] && c_year[c] >= year_lo && c_year[c] <= year_hi;
  int64_t joined = 0;
  for (int64_t i = 0; i < nb; ++i) {
    const int32_t c = b_c[i];
    if (c < 0 || (int64_t)c >= nc || !c_ok[c]) continue;
    const int32_t a = b_a[i];
    if (a < 0 || a > max_a || !a_mask[a]) continue;
    if (cnt[a] == 0 || c_year[c] < mny[a]) mny[a] = c_year[c];
    cnt[a] += 1;
    joined += 1;
  }
  int64_t ng = 0;
  for (int64_t a = 0; a < a_cap; ++a) ng += (cnt[a] > 0);
  grp_entry* g = (grp_entry*)malloc(sizeof(grp_entry) * (size_t)(ng > 0 ? ng : 1));
  int64_t j = 0;
  for (int64_t a = 0; a < a_cap; ++a)
    if (cnt[a] > 0) {
      g[j].key = (int32_t)a;
      g[j].min_year = mny[a];
      g[j].count = cnt[a];
      ++j;
    }
  int rc = radix_sort_groups(g, ng);
  const int64_t nout = ng < k ? ng : k;
  for (int64_t i = 0; i < nout && rc == 0; ++i) {
    out_key[i] = g[i].key;
    out_count[i] = g[i].count;
    out_min_year[i] = g[i].min_year;
  }
  free(a_mask);
  free(c_ok);
  free(cnt);
  free(mny);
  free(g);
  if (joined_rows) *joined_rows = joined;
  return rc ? rc : ng;
}

/* Exact distinct count of qualifying group keys (the exact-count pre-pass the
 * plain form sizes its group table with). */
int64_t oracle_distinct_groups(const int32_t* a_ids, int64_t na, const int32_t* b_a, const int32_t* b_c,
                               int64_t nb, const uint16_t* c_cat, const int32_t* c_year, int64_t nc,
                               const uint16_t* cat_set, int32_t n_cat, int32_t year_lo, int32_t year_hi) {
  int64_t joined = 0;
  return oracle_groupby_topk(a_ids, na, b_a, b_c, nb, c_cat, c_year, nc, cat_set, n_cat, year_lo, year_hi, 0, 0,
                             0, 0, &joined);
}

/* Stable LSD radix sort of (key64, value) pairs ascending by key, 8-bit
 * digits -- the checker for the GPU onesweep sort. */
int oracle_radix_sort_pairs(uint64_t* keys, uint32_t* vals, int64_t n) {
  if (n < 2) return 0;
  uint64_t* tk = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  uint32_t* tv = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
  if (!tk || !tv) {
    free(tk);
    free(tv);
    return -2;
  }
  uint64_t* sk = keys;
  uint32_t* sv = vals;
  uint64_t* dk = tk;
  uint32_t* dv = tv;
  for (int pass = 0; pass < 8; ++pass) {
    uint64_t counts[256];
    memset(counts, 0, sizeof(counts));
    const int shift = 8 * pass;
    for (int64_t i = 0; i < n; ++i) counts[(sk[i] >> shift) & 0xff] += 1;
    uint64_t sum = 0;
    for (int d = 0; d < 256; ++d) {
      const uint64_t c = counts[d];
      counts[d] = sum;
      sum += c;
    }
    for (int64_t i = 0; i < n; ++i) {
      const uint64_t pos = counts[(sk[i] >> shift) & 0xff]++;
      dk[pos] = sk[i];
      dv[pos] = sv[i];
    }
    uint64_t* t1 = sk;
    sk = dk;
    dk = t1;
    uint32_t* t2 = sv;
    sv = dv;
    dv = t2;
  }
  free(tk);
  free(tv);
  return 0;
}
