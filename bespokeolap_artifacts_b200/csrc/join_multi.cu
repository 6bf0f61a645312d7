// Shared filtered joins: up to 32 joins of the same build and probe tables
// that differ only in their predicate constants (date_lt, segment_eq), in one
// pass over each table -- the serving loop's answer to many concurrent join
// requests over the same device-resident tables, where every solo join would
// stream the same probe side again.  No reference counterpart (the reference
// runs one query per call, bespoke_tpch/query_impl.cpp:159-388); each query's
// result equals the solo filtered join (join.cu), which restates the filtered
// join of run_q3 (bespoke_tpch/query_q3.cpp:182-260).
//
// The queries are sorted by date_lt, so the queries a build row qualifies for
// are "its segment's queries" AND "the queries with date_lt > date" -- a
// suffix of the sorted order.  With j = the number of date_lt <= date:
//   mask(row) = segmask[segment] & (~0u << j)
//   count   one pass: histogram of (segment, j) per block; the last block turns
//           it into each query's qualifying-row count and the union count
//           (rows with a non-empty mask), which sizes the table on the device;
//   init    clears the table for the union and the Bloom filter;
//   build   one pass: rows with a non-empty mask insert (key << 32 | mask) with
//           a 64-bit CAS; a key that is already present (two build rows with
//           one key) cannot carry per-query multiplicities in one word, so it
//           marks the whole call for an exact solo rerun of every query;
//   probe   one pass: Bloom filter in shared memory (TMA bulk copy), the warp
//           queue of candidates, table lookups, then per candidate the mask of
//           queries it joins for; per round, for every query present in the
//           warp, the warp reduces (count, T, rr) with redux.sync and lane k
//           keeps query k's 64-bit totals; blocks add them into 128-bit totals
//           and the last block writes every query's result.
#include <algorithm>
#include <numeric>

#include "common.cuh"
#include "rows.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kMq = BO_JOIN_MULTI_MAX;  // queries per call (one mask bit each)
constexpr int kMqBlock = 512;
constexpr int kMqBuildBlock = 256;
constexpr int kMqRowsPerLane = 8;       // probe rows per lane per warp step
constexpr int kMqBuildRows = 16;        // build rows per thread
constexpr int kMqWarps = kMqBlock / 32;
constexpr int kMqMinCapLog2 = 10;

// Predicate constants, queries in date_lt order (sorted index k = mask bit k).
struct MultiQ {
  int32_t n;
  int32_t n_seg;                 // distinct segments among the queries
  int32_t date_lt[kMq];          // ascending
  uint32_t seg_of[kMq];          // compact segment of sorted query k
  uint32_t segmask[kMq];         // queries of compact segment i
  int32_t perm[kMq];             // caller's index of sorted query k
  int16_t seg_idx[256];          // segment byte -> compact segment or -1
};

// Device state of one call ("join_multi_meta" region; cleared by the host
// before every call).
struct MqState {
  unsigned long long hist[kMq * (kMq + 1)];  // [compact segment][j]
  unsigned long long count[kMq];             // qualifying rows per sorted query
  unsigned long long acc[kMq * 6];           // per query 128-bit match count, sum T, sum rr
  unsigned long long distinct;
  uint32_t ticket_count, ticket_probe, dup, overflow;
  int32_t cap_log2;
  float union_rows;
};

__device__ __forceinline__ uint32_t mq_first_above(const int32_t* date_lt, int n, int32_t date) {
  uint32_t lo = 0, hi = (uint32_t)n;  // first sorted query with date_lt > date
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (date_lt[mid] > date) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

__device__ __forceinline__ uint32_t mq_suffix(uint32_t j) { return j >= 32u ? 0u : (~0u << j); }

__device__ __forceinline__ uint32_t mq_mask(const MultiQ& q, int32_t date, uint32_t seg_byte) {
  const int idx = q.seg_idx[seg_byte & 0xffu];
  if (idx < 0) return 0u;
  return q.segmask[idx] & mq_suffix(mq_first_above(q.date_lt, q.n, date));
}

// --------------------------------------------------------------- count ---
__global__ void __launch_bounds__(kMqBuildBlock) mq_count_kernel(bo_join_build_cols b, MultiQ qv, MqState* st) {
  __shared__ MultiQ q;
  __shared__ uint32_t h[kMq * (kMq + 1)];
  if (threadIdx.x == 0) q = qv;
  for (int i = threadIdx.x; i < kMq * (kMq + 1); i += kMqBuildBlock) h[i] = 0;
  __syncthreads();
  const int64_t n = b.n_rows;
  for (int64_t i = (int64_t)blockIdx.x * kMqBuildBlock + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * kMqBuildBlock) {
    const int idx = q.seg_idx[b.segment[i]];
    if (idx < 0) continue;
    atomicAdd(h + idx * (kMq + 1) + mq_first_above(q.date_lt, q.n, b.date[i]), 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < q.n_seg * (kMq + 1); i += kMqBuildBlock)
    if (h[i]) atomicAdd(st->hist + i, (unsigned long long)h[i]);
  if (last_block(&st->ticket_count) && threadIdx.x == 0) {
    // query k (segment s = seg_of[k]) counts the rows of segment s with j <= k
    for (int k = 0; k < q.n; ++k) {
      unsigned long long c = 0;
      for (int j = 0; j <= k; ++j) c += __ldcg(st->hist + q.seg_of[k] * (kMq + 1) + j);
      st->count[k] = c;
    }
    unsigned long long u = 0;
    for (int s = 0; s < q.n_seg; ++s)
      for (int j = 0; j <= q.n; ++j)
        if (q.segmask[s] & mq_suffix((uint32_t)j)) u += __ldcg(st->hist + s * (kMq + 1) + j);
    st->union_rows = (float)u;
  }
}

// ---------------------------------------------------------------- init ---
__global__ void mq_init_kernel(unsigned long long* slots, uint32_t* bloom, MqState* st, int32_t max_log2) {
  const double want = (double)st->union_rows * 2.0;  // exact count: load <= 0.5
  int32_t cl = kMqMinCapLog2;
  while (cl < max_log2 && (double)(1ull << cl) < want) ++cl;
  const uint64_t cap = 1ull << cl;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  ulonglong2* s2 = reinterpret_cast<ulonglong2*>(slots);
  for (uint64_t i = tid; i < cap / 2; i += stride) s2[i] = make_ulonglong2(kEmptySlot, kEmptySlot);
  uint4* b4 = reinterpret_cast<uint4*>(bloom);
  for (uint64_t i = tid; i < kBloomWords / 4; i += stride) b4[i] = make_uint4(0, 0, 0, 0);
  if (tid == 0) st->cap_log2 = cl;
}

// --------------------------------------------------------------- build ---
__device__ __forceinline__ void mq_insert(unsigned long long* slots, uint32_t* bloom, uint64_t mask, int32_t key,
                                          uint32_t qmask, uint32_t& newkeys, uint32_t& dup, uint32_t& full) {
  uint64_t idx = hash32((uint32_t)key) & mask;
  const unsigned long long mine = ((unsigned long long)(uint32_t)key << 32) | qmask;
  for (uint64_t step = 0; step <= mask; ++step) {
    const unsigned long long old = atomicCAS(slots + idx, kEmptySlot, mine);
    if (old == kEmptySlot) {
      ++newkeys;
      uint32_t w, bits;
      bloom_pos((uint32_t)key, w, bits);
      atomicOr(bloom + w, bits);
      return;
    }
    if ((uint32_t)(old >> 32) == (uint32_t)key) {
      dup = 1;
      return;
    }
    idx = (idx + 1) & mask;
  }
  full = 1;
}

__global__ void __launch_bounds__(kMqBuildBlock) mq_build_kernel(bo_join_build_cols b, MultiQ qv,
                                                                 unsigned long long* slots, uint32_t* bloom,
                                                                 MqState* st) {
  __shared__ MultiQ q;
  __shared__ uint32_t queue[kMqBuildBlock / 32][2][32 * kMqBuildRows];
  if (threadIdx.x == 0) q = qv;
  __syncthreads();
  const uint64_t mask = (1ull << __ldcg(&st->cap_log2)) - 1;
  const int lane = threadIdx.x & 31;
  uint32_t* qk = queue[threadIdx.x >> 5][0];
  uint32_t* qm = queue[threadIdx.x >> 5][1];
  uint32_t newkeys = 0, dup = 0, full = 0;
  const int64_t n = b.n_rows;
  const int64_t steps = (n + kMqBuildRows - 1) / kMqBuildRows;
  const int64_t steps_w = (steps + 31) & ~int64_t(31);  // whole warps: the queue steps stay converged
  for (int64_t s = (int64_t)blockIdx.x * kMqBuildBlock + threadIdx.x; s < steps_w;
       s += (int64_t)gridDim.x * kMqBuildBlock) {
    const int64_t r0 = s * kMqBuildRows;
    int32_t keys[kMqBuildRows];
    uint32_t qms[kMqBuildRows];
    uint32_t any = 0;
    if (r0 + kMqBuildRows <= n) {
      const int4 sg = ld_stream_v4(b.segment + r0);
      const uint32_t sw[4] = {(uint32_t)sg.x, (uint32_t)sg.y, (uint32_t)sg.z, (uint32_t)sg.w};
      const int8v d0 = ld_stream_v8(b.date + r0), d1 = ld_stream_v8(b.date + r0 + 8);
      const int8v k0 = ld_stream_v8(b.key + r0), k1 = ld_stream_v8(b.key + r0 + 8);
#pragma unroll
      for (int k = 0; k < kMqBuildRows; ++k) {
        qms[k] = mq_mask(q, k < 8 ? d0.v[k] : d1.v[k - 8], sw[k >> 2] >> (8 * (k & 3)));
        keys[k] = k < 8 ? k0.v[k] : k1.v[k - 8];
        any |= (qms[k] != 0u) << k;
      }
    } else {
#pragma unroll
      for (int k = 0; k < kMqBuildRows; ++k) {
        qms[k] = 0;
        keys[k] = 0;
        if (r0 + k < n) {
          qms[k] = mq_mask(q, b.date[r0 + k], b.segment[r0 + k]);
          keys[k] = b.key[r0 + k];
          any |= (qms[k] != 0u) << k;
        }
      }
    }
    uint32_t total;
    uint32_t pos = warp_exclusive_scan(__popc(any), total);
    if (total == 0) continue;  // warp-uniform
#pragma unroll
    for (int k = 0; k < kMqBuildRows; ++k)
      if ((any >> k) & 1u) {
        qk[pos] = (uint32_t)keys[k];
        qm[pos] = qms[k];
        ++pos;
      }
    __syncwarp();
    for (uint32_t i = lane; i < total; i += 32) mq_insert(slots, bloom, mask, (int32_t)qk[i], qm[i], newkeys, dup, full);
    __syncwarp();
  }
  const uint32_t wn = warp_sum_u32(newkeys);
  const unsigned wd = __any_sync(0xffffffffu, dup), wf = __any_sync(0xffffffffu, full);
  if (lane == 0) {
    if (wn) atomicAdd(&st->distinct, (unsigned long long)wn);
    if (wd) atomicOr(&st->dup, 1u);
    if (wf) atomicOr(&st->overflow, 1u);
  }
}

// --------------------------------------------------------------- probe ---
// Per-lane totals of the query this lane owns (lane k <-> sorted query k).
struct MqAcc {
  unsigned long long cnt = 0, t = 0, rr = 0;
  uint32_t bad = 0;
};

// Resolves the warp's queued candidates (as probe_resolve in rows.cuh, R = 2
// per lane per round), then reduces each present query's (count, T, rr) over
// the warp; T is split in 16-bit halves so every warp sum fits 32 bits.
__device__ __forceinline__ void mq_resolve(const int32_t* qf, const uint16_t* qo, uint32_t total, int64_t base,
                                           const unsigned long long* slots, uint64_t mask, const int64_t* price,
                                           const int64_t* disc, MqAcc& acc) {
  constexpr int R = 2;
  const int lane = threadIdx.x & 31;
  for (uint32_t i0 = 0; i0 < total; i0 += 32 * R) {
    int32_t key[R];
    int64_t row[R];
    uint64_t idx[R];
    unsigned long long v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const uint32_t i = i0 + r * 32 + lane;
      const bool ok = i < total;
      key[r] = ok ? qf[i] : 0;
      row[r] = ok ? base + qo[i] : 0;
      idx[r] = hash32((uint32_t)key[r]) & mask;
      v[r] = ok ? __ldg(slots + idx[r]) : kEmptySlot;
    }
    uint32_t m[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      m[r] = 0;
      if (v[r] != kEmptySlot) {
        if ((uint32_t)(v[r] >> 32) == (uint32_t)key[r])
          m[r] = (uint32_t)v[r];
        else
          m[r] = (uint32_t)probe_slow<false>(slots, mask, idx[r], (uint32_t)key[r], ~0ull);
      }
    }
    uint32_t T[R], rr[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      T[r] = 0;
      rr[r] = 0;
      if (m[r]) {
        const uint64_t p = (uint64_t)__ldg(price + row[r]), d = (uint64_t)__ldg(disc + row[r]);
        if (p >= 0x80000000ull || d > 100u) {
          acc.bad |= kErrValueRange;
          m[r] = 0;
          continue;
        }
        const uint32_t mm = 100u - (uint32_t)d, pq = (uint32_t)p / 100u, pr = (uint32_t)p - pq * 100u;
        const uint32_t rm = pr * mm, rq = rm / 100u;
        T[r] = pq * mm + rq;
        rr[r] = rm - rq * 100u;
      }
    }
    uint32_t present = __reduce_or_sync(0xffffffffu, m[0] | m[1]);
    while (present) {
      const int k = __ffs(present) - 1;
      present &= present - 1;
      uint32_t c = 0, tl = 0, th = 0, rs = 0;
#pragma unroll
      for (int r = 0; r < R; ++r)
        if ((m[r] >> k) & 1u) {
          ++c;
          tl += T[r] & 0xffffu;
          th += T[r] >> 16;
          rs += rr[r];
        }
      c = __reduce_add_sync(0xffffffffu, c);
      tl = __reduce_add_sync(0xffffffffu, tl);
      th = __reduce_add_sync(0xffffffffu, th);
      rs = __reduce_add_sync(0xffffffffu, rs);
      if (lane == k) {
        acc.cnt += c;
        acc.t += (unsigned long long)tl + ((unsigned long long)th << 16);
        acc.rr += rs;
      }
    }
  }
}

__global__ void __launch_bounds__(kMqBlock, 2) mq_probe_kernel(bo_join_probe_cols p, const unsigned long long* slots,
                                                              const uint32_t* bloom_g, MqState* st,
                                                              bo_join_result* out, MultiQ qv, uint32_t* err) {
  extern __shared__ __align__(128) uint32_t bloom_s[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int32_t q_fk[kMqWarps][32 * kMqRowsPerLane];
  __shared__ uint16_t q_off[kMqWarps][32 * kMqRowsPerLane];
  __shared__ unsigned long long part[kMqWarps][32][3];
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_arrive_expect_tx(&bar, kBloomBytes);
    bulk_copy_g2s(bloom_s, bloom_g, kBloomBytes, &bar);
  }
  __syncthreads();
  // Without the filter (a timed-out copy) every row probes the table: same answer.
  const bool use_bloom = mbar_wait_bounded(&bar, 0, kWaitLimitNs);
  __shared__ uint32_t all_ones;
  if (threadIdx.x == 0) all_ones = 0xffffffffu;
  __syncthreads();
  const uint32_t* bl = use_bloom ? bloom_s : &all_ones;
  const uint32_t wmask = use_bloom ? (kBloomWords - 1u) : 0u;
  MqAcc acc;
  if (!use_bloom) acc.bad |= kErrSpinTimeout;
  const uint64_t mask = (1ull << __ldcg(&st->cap_log2)) - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int32_t* qf = q_fk[warp];
  uint16_t* qo = q_off[warp];
  const int64_t n = p.n_rows;
  constexpr int kStep = 32 * kMqRowsPerLane;
  const int64_t steps = (n + kStep - 1) / kStep;
  for (int64_t s = (int64_t)blockIdx.x * kMqWarps + warp; s < steps; s += (int64_t)gridDim.x * kMqWarps) {
    const int64_t base = s * kStep;
    const int64_t r0 = base + lane * kMqRowsPerLane;
    int32_t fk[kMqRowsPerLane];
    uint32_t valid = 0xffu;
    if (r0 + kMqRowsPerLane <= n) {
      const int8v f0 = ld_stream_v8(p.fk + r0);
#pragma unroll
      for (int k = 0; k < kMqRowsPerLane; ++k) fk[k] = f0.v[k];
    } else {
      valid = 0;
#pragma unroll
      for (int k = 0; k < kMqRowsPerLane; ++k) {
        fk[k] = 0;
        if (r0 + k < n) {
          fk[k] = p.fk[r0 + k];
          valid |= 1u << k;
        }
      }
    }
    uint32_t hit = 0;
#pragma unroll
    for (int k = kMqRowsPerLane - 1; k >= 0; --k) hit = (hit << 1) | bloom_test(bl, wmask, (uint32_t)fk[k]);
    hit &= valid;
    uint32_t total;
    uint32_t pos = warp_exclusive_scan(__popc(hit), total);
#pragma unroll
    for (int k = 0; k < kMqRowsPerLane; ++k)
      if ((hit >> k) & 1u) {
        qf[pos] = fk[k];
        qo[pos] = (uint16_t)(lane * kMqRowsPerLane + k);
        ++pos;
      }
    __syncwarp();
    mq_resolve(qf, qo, total, base, slots, mask, p.price, p.discount, acc);
    __syncwarp();
  }
  if (!use_bloom) mbar_wait_bounded(&bar, 0, kWaitLimitNs);  // the copy may still be in flight
  if (acc.bad) raise_error(err, acc.bad);
  part[warp][lane][0] = acc.cnt;
  part[warp][lane][1] = acc.t;
  part[warp][lane][2] = acc.rr;
  __syncthreads();
  if (threadIdx.x < 32 * 3) {
    const int k = threadIdx.x / 3, f = threadIdx.x % 3;
    unsigned long long v = 0;  // per block: < 2^32 rows x < 2^31, fits 64 bits
    for (int w = 0; w < kMqWarps; ++w) v += part[w][k][f];
    if (v) atomic_add_i128(st->acc + 6 * k + 2 * f, (__int128)v);
  }
  if (last_block(&st->ticket_probe) && threadIdx.x < qv.n) {
    const int k = threadIdx.x;
    uint32_t fbad = 0;
    const __int128 m = load_i128(st->acc + 6 * k), t = load_i128(st->acc + 6 * k + 2),
                   rr = load_i128(st->acc + 6 * k + 4);
    bo_join_result r;
    r.build_rows = (int64_t)__ldcg(&st->count[k]);
    r.distinct_keys = r.build_rows;  // no key repeats (else the call is marked for rerun)
    r.match_count = narrow_i64(m, fbad);
    r.sum_trunc = to_bo_i128(t);
    r.sum_exact = to_bo_i128(t * 100 + rr);
    r.capacity_log2 = __ldcg(&st->cap_log2);
    r.overflowed = (int32_t)(__ldcg(&st->dup) | __ldcg(&st->overflow));
    r.reruns = 0;
    r.mode = 0;
    out[qv.perm[k]] = r;
    if (fbad) raise_error(err, fbad);
  }
}

int ceil_log2_u64(uint64_t v) {
  int l = 0;
  while ((1ull << l) < v) ++l;
  return l;
}

int mq_grid(bo_ctx* ctx, const void* k, int block, size_t smem, int64_t items) {
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(k, block, smem);
  return (int)std::max<int64_t>(1, std::min<int64_t>(resident, (items + block - 1) / block));
}

int mq_check(bo_ctx* ctx, const bo_join_build_cols* b, const bo_join_probe_cols* p, const bo_join_params* prm,
             int32_t n) {
  if (!b || !p || !prm) return set_error(ctx, BO_ERR_INVALID, "join_multi: null argument");
  if (n < 1 || n > kMq) return set_error(ctx, BO_ERR_INVALID, "join_multi: %d queries (1..%d)", n, kMq);
  if (b->n_rows < 0 || p->n_rows < 0 || b->n_rows > 0x7fffffffll)
    return set_error(ctx, BO_ERR_INVALID, "join_multi: row counts");
  if (b->n_rows > 0 && (!b->key || !b->date || !b->segment || !aligned32(b->key) || !aligned32(b->date) ||
                        !aligned32(b->segment)))
    return set_error(ctx, BO_ERR_INVALID, "join_multi: build column null or not 32-byte aligned");
  if (p->n_rows > 0 && (!p->fk || !p->price || !p->discount || !aligned32(p->fk) || !aligned32(p->price) ||
                        !aligned32(p->discount)))
    return set_error(ctx, BO_ERR_INVALID, "join_multi: probe column null or not 32-byte aligned");
  for (int i = 0; i < n; ++i)
    if (prm[i].segment_eq < 0 || prm[i].segment_eq > 255)
      return set_error(ctx, BO_ERR_INVALID, "join_multi: segment_eq %d outside uint8", prm[i].segment_eq);
  return BO_OK;
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_join_multi_device(bo_ctx* ctx, const bo_join_build_cols* b, const bo_join_probe_cols* p,
                                    const bo_join_params* prm, int32_t n_queries, bo_join_result* out_device) {
  BO_CHECK_CTX(ctx);
  int rc = mq_check(ctx, b, p, prm, n_queries);
  if (rc) return rc;
  if (!out_device) return set_error(ctx, BO_ERR_INVALID, "join_multi: null output");
  // Sort the queries by date_lt (stable) and compact their segments.
  MultiQ q{};
  q.n = n_queries;
  std::vector<int> order(n_queries);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return prm[x].date_lt < prm[y].date_lt; });
  for (int i = 0; i < 256; ++i) q.seg_idx[i] = -1;
  for (int k = 0; k < n_queries; ++k) {
    const bo_join_params& x = prm[order[k]];
    q.date_lt[k] = x.date_lt;
    q.perm[k] = order[k];
    int16_t& si = q.seg_idx[x.segment_eq];
    if (si < 0) si = (int16_t)q.n_seg++;
    q.seg_of[k] = (uint32_t)si;
    q.segmask[si] |= 1u << k;
  }
  const int32_t max_log2 = std::max(kMqMinCapLog2, ceil_log2_u64((uint64_t)std::max<int64_t>(b->n_rows, 1) * 2));
  void* ptr = nullptr;
  if ((rc = region(ctx, "join_multi_slots", sizeof(unsigned long long) << max_log2, &ptr))) return rc;
  auto* slots = static_cast<unsigned long long*>(ptr);
  if ((rc = region(ctx, "join_multi_bloom", kBloomBytes, &ptr))) return rc;
  auto* bloom = static_cast<uint32_t*>(ptr);
  if ((rc = region(ctx, "join_multi_meta", sizeof(MqState), &ptr))) return rc;
  auto* st = static_cast<MqState*>(ptr);
  BO_CUDA(ctx, cudaMemsetAsync(st, 0, sizeof(MqState), ctx->stream));

  const void* kc = reinterpret_cast<const void*>(&mq_count_kernel);
  mq_count_kernel<<<mq_grid(ctx, kc, kMqBuildBlock, 0, b->n_rows), kMqBuildBlock, 0, ctx->stream>>>(*b, q, st);
  if ((rc = after_launch(ctx, "mq_count_kernel"))) return rc;
  const void* ki = reinterpret_cast<const void*>(&mq_init_kernel);
  mq_init_kernel<<<mq_grid(ctx, ki, 256, 0, (int64_t)1 << std::min(max_log2, 24)), 256, 0, ctx->stream>>>(
      slots, bloom, st, max_log2);
  if ((rc = after_launch(ctx, "mq_init_kernel"))) return rc;
  const void* kb = reinterpret_cast<const void*>(&mq_build_kernel);
  mq_build_kernel<<<mq_grid(ctx, kb, kMqBuildBlock, 0, (b->n_rows + kMqBuildRows - 1) / kMqBuildRows),
                    kMqBuildBlock, 0, ctx->stream>>>(*b, q, slots, bloom, st);
  if ((rc = after_launch(ctx, "mq_build_kernel"))) return rc;
  const void* kp = reinterpret_cast<const void*>(&mq_probe_kernel);
  static bool ready = false;
  if (!ready) {
    BO_CUDA(ctx, cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBloomBytes));
    ready = true;
  }
  const int gp = mq_grid(ctx, kp, kMqBlock, kBloomBytes, (p->n_rows + kMqRowsPerLane - 1) / kMqRowsPerLane);
  mq_probe_kernel<<<gp, kMqBlock, kBloomBytes, ctx->stream>>>(*p, slots, bloom, st, out_device, q, ctx->d_err);
  return after_launch(ctx, "mq_probe_kernel");
}

extern "C" int bo_join_multi_host(bo_ctx* ctx, const bo_join_build_cols* b, const bo_join_probe_cols* p,
                                  const bo_join_params* prm, int32_t n_queries, bo_join_result* out_host) {
  BO_CHECK_CTX(ctx);
  if (!out_host) return set_error(ctx, BO_ERR_INVALID, "join_multi: null output");
  void* dout = nullptr;
  int rc = region(ctx, "join_multi_out", sizeof(bo_join_result) * kMq, &dout);
  if (rc) return rc;
  if ((rc = bo_join_multi_device(ctx, b, p, prm, n_queries, static_cast<bo_join_result*>(dout)))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(out_host, dout, sizeof(bo_join_result) * (size_t)n_queries, cudaMemcpyDeviceToHost,
                               ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // synchronises the stream
  if ((rc = device_error_status(ctx, bits, "join_multi"))) return rc;
  if (out_host[0].overflowed) {  // repeated build keys: every query alone, exactly
    for (int i = 0; i < n_queries; ++i) {
      if ((rc = bo_join_plain(ctx, b, p, &prm[i], &out_host[i]))) return rc;
      out_host[i].reruns = 1;
    }
  }
  return BO_OK;
}
