// Skewed three-way join + high-cardinality group-by + ordered top-k (K4, with
// the K5 onesweep sort and K6 top-k of radix_sort.cu).
//
// Reference patterns this restates (no reference function computes the whole
// pipeline verbatim):
//   * dimension filters turned into dense masks and fact scans that count per
//     id with bounds checks: bespoke_ceb/query_q1a.cpp (mask builders before
//     :156, cast_info scan :503-601);
//   * group-by with a min aggregate: bespoke_ceb/query_q10a.cpp:843-856;
//   * order by count desc, id asc: bespoke_tpch/query_q10.cpp:318-372.
//
// Pipeline for  A(id)  B(a_id, c_id)  C(category, year; c_id = row index):
//   init     capacity (host exact count, or device-side from a predicted group
//            count), clear the group table, the Bloom filter and the A mask;
//   cfilter  C rows -> exact pass bitmap (one 32-row word per thread, no
//            atomics) and the passing ids into a 64 KB blocked Bloom filter;
//   amask    A ids -> bitmap over [0, a_id_max];
//   scan     B streamed 8 rows per lane (one 256-bit c_id load and one
//            256-bit a_id load, both L2 evict-first and prefetched a step
//            ahead, so no survivor waits on a scattered a_id read); the Bloom
//            filter (read through L1) rejects ~97% of rows without leaving
//            the SM; hits are compacted per warp with their a_id, checked
//            against the exact bitmap and the A mask, and only survivors load
//            the C year (late materialisation).  Survivors aggregate first
//            into a per-block shared-memory table (count, min year) so Zipf
//            heavy hitters cost one global update per block, then the block
//            flushes into a global open-addressing table (key << 32 | count
//            with 64-bit atomicCAS, min year by atomicMin).  The plain form's
//            exact pre-pass runs the same scan setting bits of a distinct
//            bitmap instead;
//   compact  occupied slots -> packed sort keys ((cmax - count) << wa | a_id)
//            with the min year as the value;
//   sort     onesweep LSD radix sort over the key bits actually used, key
//            count read from the device (no host round trip);
//   topk     first k sorted entries decoded into the result record.
#include <algorithm>

#include "common.cuh"
#include "rows.cuh"
#include "context.cuh"

namespace bo {

// The group table and the C-id Bloom filter use the join's slot and filter
// formats (rows.cuh).
constexpr unsigned long long kGbEmpty = kEmptySlot;
constexpr int kGbBloomLog2Words = kBloomLog2Words;
constexpr uint32_t kGbBloomWords = kBloomWords;
constexpr uint32_t kGbBloomBytes = kBloomBytes;
constexpr int kGbBlock = 256;
constexpr int kGbWarps = kGbBlock / 32;
constexpr int kGbRowsPerLane = 8;
constexpr int kGbRowsPerWarpStep = 32 * kGbRowsPerLane;
constexpr int kGbQueue = 384;        // per-warp candidate queue (entries)
constexpr int kGbFlushAt = 128;      // resolve once this many candidates are queued
constexpr int kGbResolveR = 4;       // independent candidates per lane per resolve round
// Per-block pre-aggregation table for Zipf heavy hitters: small (tail keys go
// straight to the global table, where they do not contend) and probed at most
// kGbLocalProbes times, so a full table costs a tail key two shared CAS.
constexpr int kGbLocalSlots = 256;
constexpr int kGbLocalProbes = 2;
constexpr int kGbMinCapLog2 = 10;
constexpr float kGbPresizeFactor = 2.5f;
constexpr int kMaxCats = 64;

struct GbMeta {
  int32_t cap_log2;
  uint32_t overflow;
  uint32_t done;
  uint32_t pad;
  unsigned long long joined;          // joined (surviving) B rows
  unsigned long long distinct;        // groups inserted into the global table
  unsigned long long n_out;           // compacted groups (sort key count)
  unsigned long long c_pass;          // qualifying C rows
  unsigned long long exact_distinct;  // plain pre-pass result
  unsigned long long inv_max;         // largest packed (cmax - count): the smallest count's
};

struct CatSet {
  uint16_t v[kMaxCats];
  int32_t n;
};

__device__ __forceinline__ int32_t gb_presize_log2(const float* pred, int32_t host_log2, int32_t max_log2) {
  if (!pred) return host_log2;
  float p = *pred;
  if (!(p >= 0.0f)) p = 0.0f;
  const double want = (double)p * kGbPresizeFactor;
  int32_t cl = kGbMinCapLog2;
  while (cl < max_log2 && (double)(1ull << cl) < want) ++cl;
  return cl;
}

// ------------------------------------------------------------------ init --
// clear_filters = 0 re-initialises only the group table (the plain form's
// second phase keeps the C bitmap, Bloom filter, A mask and filter counters).
__global__ void gb_init_kernel(unsigned long long* slots, int32_t* mins, uint32_t* bloom, uint32_t* amask,
                               uint32_t* dbits, int64_t mask_words, GbMeta* meta, const float* pred, int32_t host_log2,
                               int32_t max_log2, int clear_filters) {
  const int32_t cl = gb_presize_log2(pred, host_log2, max_log2);
  const uint64_t cap = 1ull << cl;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t i = tid; i < cap; i += stride) {
    slots[i] = kGbEmpty;
    mins[i] = 0x7fffffff;
  }
  if (clear_filters) {
    for (uint64_t i = tid; i < kGbBloomWords; i += stride) bloom[i] = 0;
    for (uint64_t i = tid; i < (uint64_t)mask_words; i += stride) {
      amask[i] = 0;
      if (dbits) dbits[i] = 0;
    }
  }
  if (tid == 0) {
    meta->cap_log2 = cl;
    meta->overflow = 0;
    meta->done = 0;
    meta->joined = 0;
    meta->distinct = 0;
    meta->n_out = 0;
    meta->inv_max = 0;
    if (clear_filters) {
      meta->c_pass = 0;
      meta->exact_distinct = 0;
    }
  }
}

// --------------------------------------------------------------- cfilter --
// Thread w owns C rows [32w, 32w+32): one full bitmap word, written with a
// plain store.  The category set lives in a shared 65536-bit mask.
__global__ void __launch_bounds__(256) gb_cfilter_kernel(bo_gb_c_cols c, CatSet cats, int32_t year_lo,
                                                         int32_t year_hi, uint32_t* __restrict__ cbits,
                                                         uint32_t* __restrict__ bloom, GbMeta* meta) {
  __shared__ uint32_t catmask[2048];
  for (int i = threadIdx.x; i < 2048; i += blockDim.x) catmask[i] = 0;
  __syncthreads();
  if (threadIdx.x < cats.n) atomicOr(&catmask[cats.v[threadIdx.x] >> 5], 1u << (cats.v[threadIdx.x] & 31u));
  __syncthreads();
  const int64_t n = c.n_rows;
  const int64_t words = (n + 31) / 32;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  uint32_t passed = 0;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += stride) {
    const int64_t r0 = w * 32;
    uint32_t bits = 0;
    if (r0 + 32 <= n) {
      int8v cat[2];
      cat[0] = ld_stream_v8(c.category + r0);
      cat[1] = ld_stream_v8(c.category + r0 + 16);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int8v y = ld_stream_v8(c.year + r0 + 8 * q);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int row = 8 * q + k;
          const uint32_t word = (uint32_t)cat[row >> 4].v[(row & 15) >> 1];
          const uint32_t cv = (row & 1) ? (word >> 16) : (word & 0xffffu);
          const bool ok = ((catmask[cv >> 5] >> (cv & 31u)) & 1u) && y.v[k] >= year_lo && y.v[k] <= year_hi;
          bits |= (uint32_t)ok << row;
        }
      }
    } else {
      for (int k = 0; k < 32 && r0 + k < n; ++k) {
        const uint32_t cv = c.category[r0 + k];
        const int32_t y = c.year[r0 + k];
        const bool ok = ((catmask[cv >> 5] >> (cv & 31u)) & 1u) && y >= year_lo && y <= year_hi;
        bits |= (uint32_t)ok << k;
      }
    }
    cbits[w] = bits;
    passed += __popc(bits);
    uint32_t b = bits;
    while (b) {
      const int k = __ffs(b) - 1;
      b &= b - 1;
      uint32_t bw, bb;
      bloom_pos((uint32_t)(r0 + k), bw, bb);
      atomicOr(bloom + bw, bb);
    }
  }
  __shared__ uint32_t part[8];
  passed = warp_sum_u32(passed);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = passed;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += part[i];
    if (t) atomicAdd(&meta->c_pass, (unsigned long long)t);
  }
}

// ----------------------------------------------------------------- amask --
__global__ void gb_amask_kernel(bo_gb_a_cols a, int32_t a_id_max, uint32_t* __restrict__ amask, uint32_t* err) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  uint32_t bad = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n_rows; i += stride) {
    const int32_t id = a.id[i];
    if (id < 0) continue;  // the reference's id masks skip negative ids
    if (id > a_id_max) {
      bad = 1;
      continue;
    }
    atomicOr(amask + (id >> 5), 1u << (id & 31));
  }
  if (bad) raise_error(err, kErrValueRange);
}

// ------------------------------------------------------------------ scan --

// kMode 0: exact distinct pre-pass (bits of a distinct bitmap); 1: aggregate.
// Records of the radix-partitioned form: the scan appends (key, count, min
// year, partition) records to one array through a warp-aggregated cursor (so
// skewed keys cannot overflow a partition's share), and a counting scatter
// then groups them by partition; the partition of a key is the top bits of
// hash32(key) (shift = 32 - log2 partitions; 32 for one partition).
struct GbParts {
  uint4* records = nullptr;
  uint32_t* cursor = nullptr;
  uint32_t cap = 0;
  uint32_t shift = 32;
  __device__ __forceinline__ uint32_t of(uint32_t key) const { return shift >= 32 ? 0u : hash32(key) >> shift; }
  __device__ __forceinline__ bool put(uint32_t pos, uint32_t key, uint32_t cnt, int32_t mn) const {
    if (pos >= cap) return false;  // more records than the prediction allowed for: the call reruns exactly
    records[pos] = make_uint4(key, cnt, (uint32_t)mn, of(key));
    return true;
  }
};

template <int kMode>
__global__ void __launch_bounds__(kGbBlock) gb_scan_kernel(bo_gb_b_cols b, int64_t n_c, int32_t a_id_max,
                                                           const uint32_t* __restrict__ bloom_g,
                                                           const uint32_t* __restrict__ cbits,
                                                           const int32_t* __restrict__ c_year,
                                                           const uint32_t* __restrict__ amask,
                                                           unsigned long long* slots, int32_t* mins, uint32_t* dbits,
                                                           GbMeta* meta, uint64_t probe_limit, GbParts parts,
                                                           uint32_t* err) {
  __shared__ int32_t q_c[kGbWarps][kGbQueue];
  __shared__ uint32_t q_row[kGbWarps][kGbQueue];
  __shared__ uint32_t l_key[kGbLocalSlots];
  __shared__ uint32_t l_cnt[kGbLocalSlots];
  __shared__ int32_t l_min[kGbLocalSlots];
  __shared__ uint32_t red[3][kGbWarps];
  for (int i = threadIdx.x; i < kGbLocalSlots; i += blockDim.x) {
    l_key[i] = 0xffffffffu;
    l_cnt[i] = 0;
    l_min[i] = 0x7fffffff;
  }
  __syncthreads();
  uint32_t bad = 0;
  // The Bloom filter is read through L1 (64 KB, shared by the SM's CTAs) rather
  // than copied into every CTA's shared memory: registers then allow 3 CTAs
  // per SM instead of 2 (measured ~8% faster per query than the staged copy).
  const uint32_t* bl = bloom_g;
  const uint32_t wmask = kGbBloomWords - 1u;
  const int32_t cl = kMode ? __ldg(&meta->cap_log2) : 0;
  const uint64_t mask = (1ull << cl) - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int32_t* qc = q_c[warp];
  uint32_t* qr = q_row[warp];
  uint32_t qn = 0;  // queued candidates (warp-uniform)
  uint32_t joined = 0, newkeys = 0, full = 0;
  const int64_t n = b.n_rows;
  const int64_t steps = (n + kGbRowsPerWarpStep - 1) / kGbRowsPerWarpStep;
  const int64_t nwarps = (int64_t)gridDim.x * kGbWarps;
  // One step of software prefetch: the next step's c_ids are in flight while
  // the current step is tested and resolved.
  auto load_step = [&](int64_t st, int32_t (&out)[kGbRowsPerLane], int32_t (&out_a)[kGbRowsPerLane], uint32_t& vmask) {
    const int64_t r0 = st * kGbRowsPerWarpStep + lane * kGbRowsPerLane;
    vmask = 0;
    if (st >= steps) return;
    if (r0 + kGbRowsPerLane <= n) {
      const int8v c0 = ld_first_v8(b.c_id + r0);
      const int8v a0 = ld_first_v8(b.a_id + r0);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        out[k] = c0.v[k];
        out_a[k] = a0.v[k];
      }
      vmask = 0xffu;
    } else {
#pragma unroll
      for (int k = 0; k < kGbRowsPerLane; ++k) {
        out[k] = -1;
        out_a[k] = -1;
        if (r0 + k < n) {
          out[k] = b.c_id[r0 + k];
          out_a[k] = b.a_id[r0 + k];
          vmask |= 1u << k;
        }
      }
    }
  };
  // Resolves the warp's queued candidates: lanes take up to kGbResolveR
  // entries each and every round issues its loads for all of them at once
  // (exact C bitmap; then the C year of the passing ones; then the A mask),
  // so a warp has many independent memory chains in flight.  The queue holds
  // each candidate's c_id and a_id.
  auto resolve = [&](uint32_t cnt) {
    __syncwarp();
    for (uint32_t i0 = 0; i0 < cnt; i0 += 32 * kGbResolveR) {
      int32_t c[kGbResolveR];
      uint32_t row[kGbResolveR], w[kGbResolveR];
      int32_t a[kGbResolveR], y[kGbResolveR];
#pragma unroll
      for (int r = 0; r < kGbResolveR; ++r) {
        const uint32_t i = i0 + r * 32 + lane;
        c[r] = i < cnt ? qc[i] : -1;
        row[r] = i < cnt ? qr[i] : 0u;  // the candidate's a_id
        const bool in = (uint32_t)c[r] < (uint32_t)n_c;  // negative or past C: no partner
        w[r] = in ? __ldg(cbits + (c[r] >> 5)) : 0u;
      }
#pragma unroll
      for (int r = 0; r < kGbResolveR; ++r) {
        const bool pass = (w[r] >> (c[r] & 31)) & 1u;
        a[r] = pass ? (int32_t)row[r] : -1;
        y[r] = (pass && kMode >= 1) ? __ldg(c_year + c[r]) : 0;
      }
      // Survivors: A-mask test, then the heavy-hitter table in shared memory;
      // the rest try their first global slot with one CAS each, all issued
      // before any result is used (collisions continue out of line).
      bool pend[kGbResolveR];
#pragma unroll
      for (int r = 0; r < kGbResolveR; ++r) {
        const bool in_a = a[r] >= 0 && a[r] <= a_id_max;
        const uint32_t m = in_a ? __ldg(amask + (a[r] >> 5)) : 0u;
        pend[r] = false;
        if (!in_a || !((m >> (a[r] & 31)) & 1u)) continue;
        ++joined;
        if (kMode == 0) {
          atomicOr(dbits + (a[r] >> 5), 1u << (a[r] & 31));
          continue;
        }
        const uint32_t h = hash32((uint32_t)a[r]);
        bool done = false;
#pragma unroll 1
        for (int p = 0; p < kGbLocalProbes && !done; ++p) {
          const int sl = (int)((h + p) & (kGbLocalSlots - 1));
          const uint32_t old = atomicCAS(&l_key[sl], 0xffffffffu, (uint32_t)a[r]);
          if (old == 0xffffffffu || old == (uint32_t)a[r]) {
            atomicAdd(&l_cnt[sl], 1u);
            atomicMin(&l_min[sl], y[r]);
            done = true;
          }
        }
        pend[r] = !done;
      }
      if (kMode == 2) {
        // Partitioned form: each survivor appends a (key, 1, year) record;
        // the warp reserves its records with one atomic per round.
#pragma unroll
        for (int r = 0; r < kGbResolveR; ++r) {
          const uint32_t pm = __ballot_sync(0xffffffffu, pend[r]);
          if (!pm) continue;  // warp-uniform
          const int leader = __ffs(pm) - 1;
          uint32_t first_pos = 0;
          if (lane == leader) first_pos = atomicAdd(parts.cursor, (uint32_t)__popc(pm));
          first_pos = __shfl_sync(0xffffffffu, first_pos, leader);
          if (pend[r] && !parts.put(first_pos + __popc(pm & ((1u << lane) - 1u)), (uint32_t)a[r], 1u, y[r]))
            full = 1;
        }
      }
      if (kMode == 1) {
        unsigned long long got[kGbResolveR];
        uint64_t first[kGbResolveR];
#pragma unroll
        for (int r = 0; r < kGbResolveR; ++r) {
          first[r] = pend[r] ? (hash32((uint32_t)a[r]) & mask) : 0;
          got[r] = pend[r] ? atomicCAS(slots + first[r], kGbEmpty, (unsigned long long)(uint32_t)a[r] << 32)
                           : 0ull;
        }
#pragma unroll
        for (int r = 0; r < kGbResolveR; ++r) {
          if (!pend[r]) continue;
          if (got[r] == kGbEmpty) ++newkeys;
          if (got[r] == kGbEmpty || (uint32_t)(got[r] >> 32) == (uint32_t)a[r]) {
            atomicAdd(slots + first[r], 1ull);
            atomicMin(mins + first[r], y[r]);
          } else if (!gb_global_insert(slots, mins, mask, (uint32_t)a[r], 1u, y[r], newkeys, (first[r] + 1) & mask,
                                              probe_limit)) {
            full = 1;
          }
        }
      }
    }
    __syncwarp();
  };
  int32_t nxt[kGbRowsPerLane], nxt_a[kGbRowsPerLane];
  uint32_t nxt_valid;
  int64_t st = (int64_t)blockIdx.x * kGbWarps + warp;
  load_step(st, nxt, nxt_a, nxt_valid);
  for (; st < steps; st += nwarps) {
    const int64_t base = st * kGbRowsPerWarpStep;
    int32_t cid[kGbRowsPerLane], aid[kGbRowsPerLane];
#pragma unroll
    for (int k = 0; k < kGbRowsPerLane; ++k) {
      cid[k] = nxt[k];
      aid[k] = nxt_a[k];
    }
    const uint32_t valid = nxt_valid;
    load_step(st + nwarps, nxt, nxt_a, nxt_valid);
    // Branch-free Bloom test of all 8 rows (every lookup is issued; without
    // the filter every word reads as all ones).
    // (The c_id range check happens in the rare resolve path below.)
    uint32_t hit = 0;
#pragma unroll
    for (int k = kGbRowsPerLane - 1; k >= 0; --k) {
      const uint32_t h = (uint32_t)cid[k] * 0x9E3779B1u;
      const uint32_t x = __ldg(bl + ((h >> (32 - kGbBloomLog2Words)) & wmask));
      hit = (hit << 1) | (__funnelshift_r(x, x, h) & __funnelshift_r(x, x, h >> 5) & 1u);
    }
    hit &= valid;
#pragma unroll
    for (int half = 0; half < 1; ++half) {
      const uint32_t hm = (hit >> (8 * half)) & 0xffu;
      uint32_t total;
      uint32_t pos = warp_exclusive_scan(__popc(hm), total);
      if (total == 0) continue;  // warp-uniform
      if (qn + total > kGbQueue) {  // keep room: resolve what is queued first
        resolve(qn);
        qn = 0;
      }
      pos += qn;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if ((hm >> k) & 1u) {
          qc[pos] = cid[8 * half + k];
          qr[pos] = (uint32_t)aid[8 * half + k];
          ++pos;
        }
      }
      qn += total;
      __syncwarp();
      if (qn >= kGbFlushAt) {
        resolve(qn);
        qn = 0;
      }
    }
  }
  if (qn) resolve(qn);
  __syncthreads();
  if (kMode == 1) {
    // Flush the block's pre-aggregated groups into the global table.
    for (int i = threadIdx.x; i < kGbLocalSlots; i += blockDim.x) {
      if (l_key[i] != 0xffffffffu)
        if (!gb_global_insert(slots, mins, mask, l_key[i], l_cnt[i], l_min[i], newkeys, ~0ull, probe_limit))
          full = 1;
    }
  } else if (kMode == 2) {
    // ... or as records, one per pre-aggregated group.
    for (int i = threadIdx.x; i < kGbLocalSlots; i += blockDim.x) {
      if (l_key[i] != 0xffffffffu)
        if (!parts.put(atomicAdd(parts.cursor, 1u), l_key[i], l_cnt[i], l_min[i])) full = 1;
    }
  }
  if (bad) raise_error(err, bad);
  const uint32_t wj = warp_sum_u32(joined), wn = warp_sum_u32(newkeys);
  const unsigned wf = __any_sync(0xffffffffu, full != 0);
  if (lane == 0) {
    red[0][warp] = wj;
    red[1][warp] = wn;
    red[2][warp] = wf;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tj = 0, tn = 0, tf = 0;
    for (int w = 0; w < kGbWarps; ++w) {
      tj += red[0][w];
      tn += red[1][w];
      tf |= red[2][w];
    }
    if (tj) atomicAdd(&meta->joined, (unsigned long long)tj);
    if (tn) {
      const unsigned long long before = atomicAdd(&meta->distinct, (unsigned long long)tn);
      if (kMode == 1 && before + tn > (mask + 1) - ((mask + 1) >> 3)) atomicOr(&meta->overflow, 1u);
    }
    if (tf) atomicOr(&meta->overflow, 1u);
  }
}

__global__ void gb_popcount_kernel(const uint32_t* __restrict__ dbits, int64_t words, GbMeta* meta) {
  uint32_t c = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) c += __popc(dbits[i]);
  c = warp_sum_u32(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(&meta->exact_distinct, (unsigned long long)c);
}

// --------------------------------------------------------------- compact --
// Each block compacts a contiguous range of slots: warps count their occupied
// slots, one atomic per block reserves the block's output range (per-warp
// atomics on the single counter would serialise in L2).
constexpr int kCompactBlock = 256;
constexpr int kCompactPerThread = 8;

__global__ void __launch_bounds__(kCompactBlock) gb_compact_kernel(const unsigned long long* __restrict__ slots,
                                                                   const int32_t* __restrict__ mins, GbMeta* meta,
                                                                   int wa, unsigned long long cmax,
                                                                   unsigned long long* __restrict__ keys,
                                                                   uint32_t* __restrict__ vals) {
  __shared__ uint32_t warp_off[kCompactBlock / 32 + 1];
  __shared__ unsigned long long block_base;
  const int32_t cl = __ldg(&meta->cap_log2);
  const uint64_t cap = 1ull << cl;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t span = (uint64_t)kCompactBlock * kCompactPerThread;
  for (uint64_t b0 = (uint64_t)blockIdx.x * span; b0 < cap; b0 += (uint64_t)gridDim.x * span) {
    uint32_t occ = 0;
    unsigned long long v[kCompactPerThread];
#pragma unroll
    for (int j = 0; j < kCompactPerThread; ++j) {
      const uint64_t i = b0 + (uint64_t)j * kCompactBlock + threadIdx.x;
      v[j] = i < cap ? slots[i] : kGbEmpty;
      occ += v[j] != kGbEmpty;
    }
    uint32_t wtot;
    const uint32_t mine = warp_exclusive_scan(occ, wtot);
    if (lane == 0) warp_off[warp] = wtot;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t t = 0;
      for (int w = 0; w < kCompactBlock / 32; ++w) {
        const uint32_t c = warp_off[w];
        warp_off[w] = t;
        t += c;
      }
      block_base = t ? atomicAdd(&meta->n_out, (unsigned long long)t) : 0ull;
    }
    __syncthreads();
    unsigned long long pos = block_base + warp_off[warp] + mine;
    unsigned long long cmaxc = 0;  // largest count seen by this thread
#pragma unroll
    for (int j = 0; j < kCompactPerThread; ++j) {
      if (v[j] != kGbEmpty) {
        const uint64_t i = b0 + (uint64_t)j * kCompactBlock + threadIdx.x;
        const unsigned long long cnt = v[j] & 0xffffffffull;
        cmaxc = cnt > cmaxc ? cnt : cmaxc;
        keys[pos] = ((cmax - cnt) << wa) | (v[j] >> 32);
        vals[pos] = (uint32_t)mins[i];
        ++pos;
      }
    }
    // The select digit of the top-k must sit below the highest bit that
    // differs among the packed counts: track the largest count.
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, cmaxc, o);
      cmaxc = other > cmaxc ? other : cmaxc;
    }
    if (lane == 0 && cmaxc) atomicMax(&meta->inv_max, cmaxc);
    __syncthreads();
  }
}

// ------------------------------------------------- partitioned aggregate --
// Counting scatter of the records by partition (histogram, exclusive scan,
// scatter), then one block per partition (grid-stride over partitions): the
// partition's records aggregate in a shared-memory table (key, count, min
// year) and its groups are written as packed sort keys like
// gb_compact_kernel's.  A partition with more groups than the table holds
// sets the overflow flag (the caller reruns exactly).
constexpr int kPartBlock = 512;
constexpr int kPartSlots = 8192;  // slots of a partition's shared table
constexpr uint32_t kPartMaxGroups = kPartSlots / 8 * 7;  // fuller counts as overflow
constexpr int kPartProbes = 256;  // probe-chain bound: a longer chain counts as overflow
constexpr size_t kPartSmem = (size_t)kPartSlots * 12;
constexpr int kPartScanBlock = 1024;

__global__ void __launch_bounds__(kPartBlock) gb_part_hist_kernel(GbParts parts, uint32_t n_parts,
                                                                  uint32_t* __restrict__ counts) {
  extern __shared__ uint32_t hist[];
  for (uint32_t i = threadIdx.x; i < n_parts; i += kPartBlock) hist[i] = 0;
  __syncthreads();
  const uint32_t n = min(__ldcg(parts.cursor), parts.cap);
  for (uint32_t i = blockIdx.x * kPartBlock + threadIdx.x; i < n; i += gridDim.x * kPartBlock)
    atomicAdd(hist + parts.records[i].w, 1u);
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n_parts; i += kPartBlock)
    if (hist[i]) atomicAdd(counts + i, hist[i]);
}

// offsets[p] = records before partition p (offsets[n_parts] = all); fill = offsets.
__global__ void __launch_bounds__(kPartScanBlock) gb_part_scan_kernel(const uint32_t* __restrict__ counts,
                                                                      uint32_t n_parts, uint32_t* __restrict__ offsets,
                                                                      uint32_t* __restrict__ fill) {
  __shared__ uint32_t warp_tot[kPartScanBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t per = (n_parts + kPartScanBlock - 1) / kPartScanBlock;
  const uint32_t lo = threadIdx.x * per, hi = min(lo + per, n_parts);
  uint32_t local = 0;
  for (uint32_t i = lo; i < hi; ++i) local += counts[i];
  uint32_t wt;
  const uint32_t wex = warp_exclusive_scan(local, wt);
  if (lane == 0) warp_tot[warp] = wt;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kPartScanBlock / 32; ++w) {
      const uint32_t x = warp_tot[w];
      warp_tot[w] = t;
      t += x;
    }
    offsets[n_parts] = t;
  }
  __syncthreads();
  uint32_t run = warp_tot[warp] + wex;
  for (uint32_t i = lo; i < hi; ++i) {
    offsets[i] = run;
    fill[i] = run;
    run += counts[i];
  }
}

// Records -> their partition's range; the lanes of one partition reserve
// their slots with one atomic (match_any groups them).
__global__ void __launch_bounds__(kPartBlock) gb_part_scatter_kernel(GbParts parts, uint32_t* __restrict__ fill,
                                                                     uint4* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const uint32_t n = min(__ldcg(parts.cursor), parts.cap);
  const uint32_t warps = gridDim.x * (kPartBlock / 32);
  for (uint32_t i0 = (blockIdx.x * kPartBlock + threadIdx.x) & ~31u; i0 < n; i0 += warps * 32) {
    const uint32_t i = i0 + lane;
    const bool valid = i < n;
    const uint4 r = valid ? parts.records[i] : make_uint4(0, 0, 0, 0xffffffffu);
    const uint32_t peers = __match_any_sync(0xffffffffu, r.w);
    const int leader = __ffs(peers) - 1;
    uint32_t first_pos = 0;
    if (valid && lane == leader) first_pos = atomicAdd(fill + r.w, (uint32_t)__popc(peers));
    first_pos = __shfl_sync(0xffffffffu, first_pos, leader);
    if (valid) out[first_pos + __popc(peers & ((1u << lane) - 1u))] = r;
  }
}

__global__ void __launch_bounds__(kPartBlock) gb_part_agg_kernel(const uint4* __restrict__ recs,
                                                                 const uint32_t* __restrict__ offsets, int n_parts,
                                                                 GbMeta* meta, int wa, unsigned long long cmax,
                                                                 unsigned long long* __restrict__ keys,
                                                                 uint32_t* __restrict__ vals) {
  extern __shared__ __align__(16) uint32_t part_smem[];
  uint32_t* t_key = part_smem;
  uint32_t* t_cnt = part_smem + kPartSlots;
  int32_t* t_min = reinterpret_cast<int32_t*>(part_smem + 2 * kPartSlots);
  __shared__ uint32_t warp_off[kPartBlock / 32];
  __shared__ unsigned long long base;
  __shared__ uint32_t full_s, used_s;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kPer = kPartSlots / kPartBlock;
  unsigned long long cmaxc = 0;
  for (int p = blockIdx.x; p < n_parts; p += gridDim.x) {
    for (int i = threadIdx.x; i < kPartSlots; i += kPartBlock) {
      t_key[i] = 0xffffffffu;
      t_cnt[i] = 0;
      t_min[i] = 0x7fffffff;
    }
    if (threadIdx.x == 0) full_s = used_s = 0;
    __syncthreads();
    const uint32_t b0 = offsets[p], b1 = offsets[p + 1];
    for (uint32_t i = b0 + threadIdx.x; i < b1; i += kPartBlock) {
      if (*reinterpret_cast<volatile uint32_t*>(&full_s)) break;  // the call reruns: stop early
      const uint4 r = recs[i];
      uint32_t sl = hash32(r.x) & (kPartSlots - 1);
      bool done = false;
      for (int step = 0; step < kPartProbes && !done; ++step) {
        const uint32_t old = atomicCAS(t_key + sl, 0xffffffffu, r.x);
        if (old == 0xffffffffu || old == r.x) {
          if (old == 0xffffffffu && atomicAdd(&used_s, 1u) + 1u > kPartMaxGroups) full_s = 1;
          atomicAdd(t_cnt + sl, r.y);
          atomicMin(t_min + sl, (int32_t)r.z);
          done = true;
        }
        sl = (sl + 1) & (kPartSlots - 1);
      }
      if (!done) full_s = 1;
    }
    __syncthreads();
    // Emit the partition's groups: one reservation per block.
    uint32_t occ = 0;
#pragma unroll
    for (int j = 0; j < kPer; ++j) occ += t_key[j * kPartBlock + threadIdx.x] != 0xffffffffu;
    uint32_t wtot;
    const uint32_t mine = warp_exclusive_scan(occ, wtot);
    if (lane == 0) warp_off[warp] = wtot;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t t = 0;
      for (int w = 0; w < kPartBlock / 32; ++w) {
        const uint32_t x = warp_off[w];
        warp_off[w] = t;
        t += x;
      }
      base = t ? atomicAdd(&meta->n_out, (unsigned long long)t) : 0ull;
      if (t) atomicAdd(&meta->distinct, (unsigned long long)t);
      if (full_s) atomicOr(&meta->overflow, 1u);
    }
    __syncthreads();
    unsigned long long pos = base + warp_off[warp] + mine;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int i = j * kPartBlock + threadIdx.x;
      if (t_key[i] != 0xffffffffu) {
        const unsigned long long cnt = t_cnt[i];
        cmaxc = cnt > cmaxc ? cnt : cmaxc;
        keys[pos] = ((cmax - cnt) << wa) | t_key[i];
        vals[pos] = (uint32_t)t_min[i];
        ++pos;
      }
    }
    __syncthreads();
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, cmaxc, o);
    cmaxc = other > cmaxc ? other : cmaxc;
  }
  if (lane == 0 && cmaxc) atomicMax(&meta->inv_max, cmaxc);
}

// ------------------------------------------------------------------ topk --
__global__ void gb_topk_kernel(const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ vals,
                               GbMeta* meta, int k, int wa, unsigned long long cmax, int mode,
                               bo_gb_result* __restrict__ out) {
  const unsigned long long n = __ldcg(&meta->n_out);
  const int t = threadIdx.x;
  if (t < k && (unsigned long long)t < n) {
    const unsigned long long key = keys[t];
    bo_gb_row r;
    r.a_id = (int32_t)(key & ((1ull << wa) - 1ull));
    r.min_year = (int32_t)vals[t];
    r.count = (int64_t)(cmax - (key >> wa));
    out->rows[t] = r;
  }
  if (t == 0) {
    out->n_groups = (int64_t)n;
    out->joined_rows = (int64_t)__ldcg(&meta->joined);
    out->c_qualifying = (int64_t)__ldcg(&meta->c_pass);
    out->capacity_log2 = __ldcg(&meta->cap_log2);
    out->overflowed = (int32_t)__ldcg(&meta->overflow);
    out->reruns = 0;
    out->mode = mode;
    out->n_rows_out = (int32_t)(n < (unsigned long long)k ? n : (unsigned long long)k);
    out->exact_distinct = (int64_t)__ldcg(&meta->exact_distinct);
  }
}

// ------------------------------------------------------------------ host --
namespace {

int bit_length(uint64_t v) {
  int b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return b;
}

struct GbWs {
  unsigned long long* slots;
  int32_t* mins;
  uint32_t* bloom;
  uint32_t* cbits;
  uint32_t* amask;
  uint32_t* dbits;
  GbMeta* meta;
  float* pred;
  unsigned long long* keys;
  uint32_t* vals;
  unsigned long long* tkeys;
  uint32_t* tvals;
  int32_t max_log2;
  int64_t mask_words;
};

int gb_workspace(bo_ctx* ctx, const bo_gb_b_cols& b, const bo_gb_c_cols& c, int32_t a_id_max, GbWs* ws) {
  const uint64_t groups_max = std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)a_id_max + 1, (uint64_t)b.n_rows));
  const int32_t max_log2 = std::max(kGbMinCapLog2, bit_length(groups_max * 2 - 1));
  const uint64_t cap = 1ull << max_log2;
  const int64_t mask_words = ((int64_t)a_id_max + 1 + 31) / 32;
  const int64_t cwords = (c.n_rows + 31) / 32;
  size_t total = 0;
  auto add = [&](size_t bytes) { total += (bytes + 255) & ~size_t(255); };
  add(8 * cap);                       // slots
  add(4 * cap);                       // mins
  add(kGbBloomBytes);                 // bloom
  add(4 * (size_t)std::max<int64_t>(cwords, 1));
  add(4 * (size_t)mask_words);        // amask
  add(4 * (size_t)mask_words);        // dbits
  add(sizeof(GbMeta) + 64);
  add(8 * cap);                       // keys
  add(4 * cap);                       // vals
  add(8 * cap);                       // tmp keys
  add(4 * cap);                       // tmp vals
  void* base = nullptr;
  int rc = region(ctx, "gb_ws", total, &base);
  if (rc) return rc;
  char* p = static_cast<char*>(base);
  ws->slots = carve<unsigned long long>(p, cap);
  ws->mins = carve<int32_t>(p, cap);
  ws->bloom = carve<uint32_t>(p, kGbBloomWords);
  ws->cbits = carve<uint32_t>(p, (size_t)std::max<int64_t>(cwords, 1));
  ws->amask = carve<uint32_t>(p, (size_t)mask_words);
  ws->dbits = carve<uint32_t>(p, (size_t)mask_words);
  char* meta_p = p;
  p += (sizeof(GbMeta) + 64 + 255) & ~size_t(255);
  ws->meta = reinterpret_cast<GbMeta*>(meta_p);
  ws->pred = reinterpret_cast<float*>(meta_p + sizeof(GbMeta));
  ws->keys = carve<unsigned long long>(p, cap);
  ws->vals = carve<uint32_t>(p, cap);
  ws->tkeys = carve<unsigned long long>(p, cap);
  ws->tvals = carve<uint32_t>(p, cap);
  ws->max_log2 = max_log2;
  ws->mask_words = mask_words;
  return BO_OK;
}

int check_gb(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b, const bo_gb_c_cols* c,
             const bo_gb_params* prm) {
  if (!a || !b || !c || !prm) return set_error(ctx, BO_ERR_INVALID, "groupby: null argument");
  if (a->n_rows < 0 || b->n_rows < 0 || c->n_rows < 0) return set_error(ctx, BO_ERR_INVALID, "groupby: negative rows");
  if (c->n_rows > 0x7fffffffll || b->n_rows > 0xffffffffll)
    return set_error(ctx, BO_ERR_INVALID, "groupby: C above 2^31 rows or B above 2^32 rows");
  if (prm->a_id_max < 0) return set_error(ctx, BO_ERR_INVALID, "groupby: a_id_max must be >= 0");
  if (prm->k < 0 || prm->k > BO_GB_MAX_K) return set_error(ctx, BO_ERR_INVALID, "groupby: k outside [0, %d]", BO_GB_MAX_K);
  if (prm->n_categories < 0 || prm->n_categories > kMaxCats || (prm->n_categories > 0 && !prm->categories))
    return set_error(ctx, BO_ERR_INVALID, "groupby: at most %d categories", kMaxCats);
  if (b->n_rows > 0 && (!b->a_id || !b->c_id || !aligned32(b->a_id) || !aligned32(b->c_id)))
    return set_error(ctx, BO_ERR_INVALID, "groupby: B columns null or not 32-byte aligned");
  if (c->n_rows > 0 && (!c->category || !c->year || !aligned32(c->category) || !aligned32(c->year)))
    return set_error(ctx, BO_ERR_INVALID, "groupby: C columns null or not 32-byte aligned");
  if (a->n_rows > 0 && !a->id) return set_error(ctx, BO_ERR_INVALID, "groupby: A column null");
  return BO_OK;
}

int grid_res(bo_ctx* ctx, const void* k, int block, size_t smem, int64_t items) {
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(k, block, smem);
  const int64_t need = (items + block - 1) / block;
  return (int)std::max<int64_t>(1, std::min(resident, need));
}

// Filters (init, C filter, A mask): common to both forms.
int gb_prepare(bo_ctx* ctx, const bo_gb_a_cols& a, const bo_gb_c_cols& c, const bo_gb_params& prm, const GbWs& ws,
               const float* pred, int32_t host_log2) {
  const void* ki = reinterpret_cast<const void*>(&gb_init_kernel);
  const int gi = grid_res(ctx, ki, 256, 0, std::max<int64_t>((int64_t)1 << std::min(ws.max_log2, 24), ws.mask_words));
  gb_init_kernel<<<gi, 256, 0, ctx->stream>>>(ws.slots, ws.mins, ws.bloom, ws.amask, ws.dbits, ws.mask_words, ws.meta,
                                              pred, host_log2, ws.max_log2, 1);
  int rc = after_launch(ctx, "gb_init_kernel");
  if (rc) return rc;
  CatSet cs{};
  cs.n = prm.n_categories;
  for (int i = 0; i < prm.n_categories; ++i) cs.v[i] = prm.categories[i];
  const int64_t cwords = (c.n_rows + 31) / 32;
  if (cwords > 0) {
    const void* kc = reinterpret_cast<const void*>(&gb_cfilter_kernel);
    const int gc = grid_res(ctx, kc, 256, 0, cwords);
    gb_cfilter_kernel<<<gc, 256, 0, ctx->stream>>>(c, cs, prm.year_lo, prm.year_hi, ws.cbits, ws.bloom, ws.meta);
    if ((rc = after_launch(ctx, "gb_cfilter_kernel"))) return rc;
  }
  if (a.n_rows > 0 && !prm.a_mask) {
    const void* ka = reinterpret_cast<const void*>(&gb_amask_kernel);
    const int ga = grid_res(ctx, ka, 256, 0, a.n_rows);
    gb_amask_kernel<<<ga, 256, 0, ctx->stream>>>(a, prm.a_id_max, ws.amask, ctx->d_err);
    if ((rc = after_launch(ctx, "gb_amask_kernel"))) return rc;
  }
  return BO_OK;
}

template <int kMode>
int gb_launch_scan(bo_ctx* ctx, const bo_gb_b_cols& b, const bo_gb_c_cols& c, const bo_gb_params& prm,
                   const GbWs& ws, uint64_t probe_limit = ~0ull, GbParts parts = GbParts{}) {
  const void* k = reinterpret_cast<const void*>(&gb_scan_kernel<kMode>);
  const int grid = grid_res(ctx, k, kGbBlock, 0, (b.n_rows + kGbRowsPerLane - 1) / kGbRowsPerLane);
  gb_scan_kernel<kMode><<<grid, kGbBlock, 0, ctx->stream>>>(
      b, c.n_rows, prm.a_id_max, ws.bloom, ws.cbits, c.year, prm.a_mask ? prm.a_mask : ws.amask, ws.slots, ws.mins,
      ws.dbits, ws.meta, probe_limit, parts, ctx->d_err);
  return after_launch(ctx, "gb_scan_kernel");
}

// Aggregate + compact + sort + top-k, asynchronous.
int gb_aggregate_order(bo_ctx* ctx, const bo_gb_b_cols& b, const bo_gb_c_cols& c, const bo_gb_params& prm,
                       const GbWs& ws, bo_gb_result* out, int32_t mode) {
  // Exact-size tables (mode 0) probe without a bound; presized ones fail fast.
  int rc = gb_launch_scan<1>(ctx, b, c, prm, ws, mode == 0 ? ~0ull : kPresizedProbeLimit);
  if (rc) return rc;
  const int wa = std::max(1, bit_length((uint64_t)prm.a_id_max));
  const int wc = std::max(1, bit_length((uint64_t)b.n_rows));
  const unsigned long long cmax = (wc >= 64) ? ~0ull : ((1ull << wc) - 1ull);
  const uint64_t cap_max = 1ull << ws.max_log2;
  const void* kc = reinterpret_cast<const void*>(&gb_compact_kernel);
  const int gc = grid_res(ctx, kc, kCompactBlock, 0, (int64_t)cap_max / kCompactPerThread);
  gb_compact_kernel<<<gc, kCompactBlock, 0, ctx->stream>>>(ws.slots, ws.mins, ws.meta, wa, cmax, ws.keys, ws.vals);
  if ((rc = after_launch(ctx, "gb_compact_kernel"))) return rc;
  // ORDER BY count desc, a_id asc LIMIT k: radix select of the k smallest
  // packed keys, then the onesweep / in-CTA LSD sort of the candidates.
  // The candidates go to the temporary buffers; the sort uses the key
  // buffers (no longer needed) as its scratch.
  // (cmax - count) for counts in [1, max_count] shares every bit above the
  // highest bit of max_count with cmax: the select digit goes just below it
  // (inv_max holds the largest count; topk_shift takes its bit length).
  if ((rc = radix_topk_pairs(ctx, ws.keys, ws.vals, (int64_t)cap_max, &ws.meta->n_out, wa + wc, prm.k, ws.tkeys,
                             ws.tvals, ws.keys, ws.vals, wa, &ws.meta->inv_max)))
    return rc;
  gb_topk_kernel<<<1, BO_GB_MAX_K, 0, ctx->stream>>>(ws.tkeys, ws.tvals, ws.meta, prm.k, wa, cmax, mode, out);
  return after_launch(ctx, "gb_topk_kernel");
}

int gb_finish(bo_ctx* ctx, bo_gb_result* host, const bo_gb_result* dev) {
  BO_CUDA(ctx, cudaMemcpyAsync(host, dev, sizeof(bo_gb_result), cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  int rc = consume_device_errors(ctx, &bits);
  if (rc) return rc;
  return device_error_status(ctx, bits, "groupby");
}

int gb_plain_impl(bo_ctx* ctx, const bo_gb_a_cols& a, const bo_gb_b_cols& b, const bo_gb_c_cols& c,
                  const bo_gb_params& prm, bo_gb_result* out_host, int32_t reruns) {
  GbWs ws;
  int rc = gb_workspace(ctx, b, c, prm.a_id_max, &ws);
  if (rc) return rc;
  if ((rc = gb_prepare(ctx, a, c, prm, ws, nullptr, kGbMinCapLog2))) return rc;
  // Exact pre-pass: distinct qualifying groups, then one host round trip.
  if ((rc = gb_launch_scan<0>(ctx, b, c, prm, ws))) return rc;
  const void* kp = reinterpret_cast<const void*>(&gb_popcount_kernel);
  const int gp = grid_res(ctx, kp, 256, 0, ws.mask_words);
  gb_popcount_kernel<<<gp, 256, 0, ctx->stream>>>(ws.dbits, ws.mask_words, ws.meta);
  if ((rc = after_launch(ctx, "gb_popcount_kernel"))) return rc;
  unsigned long long distinct = 0;
  BO_CUDA(ctx, cudaMemcpyAsync(&distinct, &ws.meta->exact_distinct, sizeof(distinct), cudaMemcpyDeviceToHost,
                               ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const int32_t cl = std::min(ws.max_log2, std::max(kGbMinCapLog2, bit_length(std::max<uint64_t>(distinct, 1) * 2 - 1)));
  // Re-initialise only the group table at the exact size; the filters stay.
  const void* ki = reinterpret_cast<const void*>(&gb_init_kernel);
  const int gi = grid_res(ctx, ki, 256, 0, (int64_t)1 << std::min(ws.max_log2, 24));
  gb_init_kernel<<<gi, 256, 0, ctx->stream>>>(ws.slots, ws.mins, ws.bloom, ws.amask, ws.dbits, ws.mask_words, ws.meta,
                                              nullptr, cl, ws.max_log2, 0);
  if ((rc = after_launch(ctx, "gb_init_kernel"))) return rc;
  void* dout = nullptr;
  if ((rc = region(ctx, "gb_out", sizeof(bo_gb_result), &dout))) return rc;
  bo_gb_result* d = static_cast<bo_gb_result*>(dout);
  if ((rc = gb_aggregate_order(ctx, b, c, prm, ws, d, 0))) return rc;
  if ((rc = gb_finish(ctx, out_host, d))) return rc;
  out_host->reruns = reruns;
  out_host->exact_distinct = (int64_t)distinct;
  if (out_host->overflowed) return set_error(ctx, BO_ERR_OVERFLOW, "groupby: exact-size table overflowed");
  return BO_OK;
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" {

int bo_groupby_topk_plain(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b, const bo_gb_c_cols* c,
                          const bo_gb_params* prm, bo_gb_result* out_host) {
  BO_CHECK_CTX(ctx);
  int rc = check_gb(ctx, a, b, c, prm);
  if (rc) return rc;
  if (!out_host) return set_error(ctx, BO_ERR_INVALID, "groupby: null output");
  return gb_plain_impl(ctx, *a, *b, *c, *prm, out_host, 0);
}

int bo_groupby_topk_presized_device(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b,
                                    const bo_gb_c_cols* c, const bo_gb_params* prm, const float* pred_groups_device,
                                    bo_gb_result* out_device) {
  BO_CHECK_CTX(ctx);
  int rc = check_gb(ctx, a, b, c, prm);
  if (rc) return rc;
  if (!pred_groups_device || !out_device) return set_error(ctx, BO_ERR_INVALID, "groupby: null prediction/output");
  GbWs ws;
  if ((rc = gb_workspace(ctx, *b, *c, prm->a_id_max, &ws))) return rc;
  if ((rc = gb_prepare(ctx, *a, *c, *prm, ws, pred_groups_device, 0))) return rc;
  return gb_aggregate_order(ctx, *b, *c, *prm, ws, out_device, 1);
}

int bo_groupby_topk_presized(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b, const bo_gb_c_cols* c,
                             const bo_gb_params* prm, const float* pred_groups_device, bo_gb_result* out_host) {
  BO_CHECK_CTX(ctx);
  if (!out_host) return set_error(ctx, BO_ERR_INVALID, "groupby: null output");
  void* dout = nullptr;
  int rc = region(ctx, "gb_out", sizeof(bo_gb_result), &dout);
  if (rc) return rc;
  bo_gb_result* d = static_cast<bo_gb_result*>(dout);
  if ((rc = bo_groupby_topk_presized_device(ctx, a, b, c, prm, pred_groups_device, d))) return rc;
  if ((rc = gb_finish(ctx, out_host, d))) return rc;
  if (out_host->overflowed) {
    if ((rc = gb_plain_impl(ctx, *a, *b, *c, *prm, out_host, 1))) return rc;
    out_host->mode = 1;
  }
  return BO_OK;
}

int bo_groupby_topk_partitioned_device(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b,
                                       const bo_gb_c_cols* c, const bo_gb_params* prm, int32_t log2_partitions,
                                       float predicted_joined_rows, bo_gb_result* out_device) {
  BO_CHECK_CTX(ctx);
  int rc = check_gb(ctx, a, b, c, prm);
  if (rc) return rc;
  if (!out_device) return set_error(ctx, BO_ERR_INVALID, "groupby: null output");
  if (log2_partitions < 0 || log2_partitions > BO_GB_MAX_LOG2_PARTITIONS)
    return set_error(ctx, BO_ERR_INVALID, "groupby: log2_partitions %d outside [0, %d]", log2_partitions,
                     BO_GB_MAX_LOG2_PARTITIONS);
  GbWs ws;
  if ((rc = gb_workspace(ctx, *b, *c, prm->a_id_max, &ws))) return rc;
  // The global group table is not used: initialise the smallest one.
  if ((rc = gb_prepare(ctx, *a, *c, *prm, ws, nullptr, kGbMinCapLog2))) return rc;
  const uint32_t n_parts = 1u << log2_partitions;
  // Records: at most one per joined row, so at most one per B row.  The
  // buffers take that bound while it stays within kRecordBoundBytes (HBM is
  // plentiful: 60M B rows need 1.9 GB for the two record arrays); beyond it
  // they are sized from the predicted joined rows with a margin and slack.
  constexpr double kRecordBoundBytes = 16.0 * (1ull << 30);
  const double bound = (double)b->n_rows + 65536.0;
  double want = bound;
  if (bound * 2 * sizeof(uint4) > kRecordBoundBytes)
    want = std::min(bound, std::max(0.0, (double)predicted_joined_rows) * 1.25 + 65536.0);
  if (want * 2 * sizeof(uint4) > (double)(64ull << 30))
    return set_error(ctx, BO_ERR_INVALID, "groupby: predicted partition records above 64 GiB");
  GbParts parts;
  parts.cap = (uint32_t)std::min(want, (double)0xfffffff0u);
  parts.shift = log2_partitions == 0 ? 32u : (uint32_t)(32 - log2_partitions);
  const size_t rec_bytes = ((size_t)parts.cap * sizeof(uint4) + 255) & ~size_t(255);
  const size_t ctr_bytes = 4 * (3 * (size_t)n_parts + 2) + 256;
  void* pbase = nullptr;
  if ((rc = region(ctx, "gb_parts", 2 * rec_bytes + ctr_bytes, &pbase))) return rc;
  char* pp = static_cast<char*>(pbase);
  parts.records = reinterpret_cast<uint4*>(pp);
  uint4* scattered = reinterpret_cast<uint4*>(pp + rec_bytes);
  uint32_t* ctr = reinterpret_cast<uint32_t*>(pp + 2 * rec_bytes);
  parts.cursor = ctr;                   // [0]
  uint32_t* counts = ctr + 1;           // [1, 1 + n_parts)
  uint32_t* offsets = counts + n_parts; // n_parts + 1
  uint32_t* fill = offsets + n_parts + 1;
  BO_CUDA(ctx, cudaMemsetAsync(ctr, 0, 4 * (1 + (size_t)n_parts), ctx->stream));
  if ((rc = gb_launch_scan<2>(ctx, *b, *c, *prm, ws, ~0ull, parts))) return rc;
  const int wa = std::max(1, bit_length((uint64_t)prm->a_id_max));
  const int wc = std::max(1, bit_length((uint64_t)b->n_rows));
  const unsigned long long cmax = (wc >= 64) ? ~0ull : ((1ull << wc) - 1ull);
  static bool ready = false;
  const void* kh = reinterpret_cast<const void*>(&gb_part_hist_kernel);
  const void* kp = reinterpret_cast<const void*>(&gb_part_agg_kernel);
  if (!ready) {
    BO_CUDA(ctx, cudaFuncSetAttribute(kh, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(4u << BO_GB_MAX_LOG2_PARTITIONS)));
    BO_CUDA(ctx, cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPartSmem));
    ready = true;
  }
  const size_t hsmem = 4 * (size_t)n_parts;
  gb_part_hist_kernel<<<ctx->num_sms * 2, kPartBlock, hsmem, ctx->stream>>>(parts, n_parts, counts);
  if ((rc = after_launch(ctx, "gb_part_hist_kernel"))) return rc;
  gb_part_scan_kernel<<<1, kPartScanBlock, 0, ctx->stream>>>(counts, n_parts, offsets, fill);
  if ((rc = after_launch(ctx, "gb_part_scan_kernel"))) return rc;
  gb_part_scatter_kernel<<<ctx->num_sms * 4, kPartBlock, 0, ctx->stream>>>(parts, fill, scattered);
  if ((rc = after_launch(ctx, "gb_part_scatter_kernel"))) return rc;
  const int gp = (int)std::min<int64_t>(n_parts, (int64_t)ctx->num_sms * occupancy_blocks(kp, kPartBlock, kPartSmem));
  gb_part_agg_kernel<<<std::max(gp, 1), kPartBlock, kPartSmem, ctx->stream>>>(scattered, offsets, (int)n_parts,
                                                                              ws.meta, wa, cmax, ws.keys, ws.vals);
  if ((rc = after_launch(ctx, "gb_part_agg_kernel"))) return rc;
  const uint64_t cap_max = 1ull << ws.max_log2;
  if ((rc = radix_topk_pairs(ctx, ws.keys, ws.vals, (int64_t)cap_max, &ws.meta->n_out, wa + wc, prm->k, ws.tkeys,
                             ws.tvals, ws.keys, ws.vals, wa, &ws.meta->inv_max)))
    return rc;
  gb_topk_kernel<<<1, BO_GB_MAX_K, 0, ctx->stream>>>(ws.tkeys, ws.tvals, ws.meta, prm->k, wa, cmax, 2, out_device);
  return after_launch(ctx, "gb_topk_kernel");
}

int bo_groupby_topk_partitioned(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b, const bo_gb_c_cols* c,
                                const bo_gb_params* prm, int32_t log2_partitions, float predicted_joined_rows,
                                bo_gb_result* out_host) {
  BO_CHECK_CTX(ctx);
  if (!out_host) return set_error(ctx, BO_ERR_INVALID, "groupby: null output");
  void* dout = nullptr;
  int rc = region(ctx, "gb_out", sizeof(bo_gb_result), &dout);
  if (rc) return rc;
  bo_gb_result* d = static_cast<bo_gb_result*>(dout);
  if ((rc = bo_groupby_topk_partitioned_device(ctx, a, b, c, prm, log2_partitions, predicted_joined_rows, d)))
    return rc;
  if ((rc = gb_finish(ctx, out_host, d))) return rc;
  if (out_host->overflowed) {
    if ((rc = gb_plain_impl(ctx, *a, *b, *c, *prm, out_host, 1))) return rc;
    out_host->mode = 2;
  }
  return BO_OK;
}

int bo_groupby_a_mask_device(bo_ctx* ctx, const bo_gb_a_cols* a, int32_t a_id_max, uint32_t* mask_device) {
  BO_CHECK_CTX(ctx);
  if (!a || !mask_device || a_id_max < 0 || a->n_rows < 0 || (a->n_rows > 0 && !a->id))
    return set_error(ctx, BO_ERR_INVALID, "groupby_a_mask: bad argument");
  const int64_t words = ((int64_t)a_id_max + 1 + 31) / 32;
  BO_CUDA(ctx, cudaMemsetAsync(mask_device, 0, sizeof(uint32_t) * (size_t)words, ctx->stream));
  if (a->n_rows == 0) return BO_OK;
  const void* ka = reinterpret_cast<const void*>(&gb_amask_kernel);
  gb_amask_kernel<<<grid_res(ctx, ka, 256, 0, a->n_rows), 256, 0, ctx->stream>>>(*a, a_id_max, mask_device,
                                                                                   ctx->d_err);
  return after_launch(ctx, "gb_amask_kernel");
}

int bo_groupby_distinct_device(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b, const bo_gb_c_cols* c,
                               const bo_gb_params* prm, int64_t* out_device) {
  BO_CHECK_CTX(ctx);
  int rc = check_gb(ctx, a, b, c, prm);
  if (rc) return rc;
  if (!out_device) return set_error(ctx, BO_ERR_INVALID, "groupby: null output");
  GbWs ws;
  if ((rc = gb_workspace(ctx, *b, *c, prm->a_id_max, &ws))) return rc;
  if ((rc = gb_prepare(ctx, *a, *c, *prm, ws, nullptr, kGbMinCapLog2))) return rc;
  if ((rc = gb_launch_scan<0>(ctx, *b, *c, *prm, ws))) return rc;
  const void* kp = reinterpret_cast<const void*>(&gb_popcount_kernel);
  gb_popcount_kernel<<<grid_res(ctx, kp, 256, 0, ws.mask_words), 256, 0, ctx->stream>>>(ws.dbits, ws.mask_words,
                                                                                          ws.meta);
  if ((rc = after_launch(ctx, "gb_popcount_kernel"))) return rc;
  // out[0] = exact distinct groups, out[1] = joined rows
  BO_CUDA(ctx, cudaMemcpyAsync(out_device, &ws.meta->exact_distinct, sizeof(int64_t), cudaMemcpyDeviceToDevice,
                               ctx->stream));
  BO_CUDA(ctx, cudaMemcpyAsync(out_device + 1, &ws.meta->joined, sizeof(int64_t), cudaMemcpyDeviceToDevice,
                               ctx->stream));
  return BO_OK;
}

}  // extern "C"
