// Filtered hash join + scalar aggregate (filtered-join shape of run_q3,
// bespoke_tpch/query_q3.cpp:182-260).
//
// Pipeline (all on the context's stream):
//   count  (K7, plain form only)  number of qualifying build rows -> host sizes
//                                  the table from the exact count;
//   init                           picks the table capacity (from the host's
//                                  exact count, or on the device from a
//                                  predicted row count), clears the slots and
//                                  the Bloom filter;
//   build  (K2)                    filter build rows, insert keys with 64-bit
//                                  atomicCAS into open-addressing slots
//                                  (key << 32 | multiplicity), set 2 bits of a
//                                  blocked Bloom filter per new key;
//   probe  (K3)                    each block stages the 64 KB Bloom filter into
//                                  shared memory with one TMA bulk copy; probe
//                                  rows stream in 8 per lane (one 256-bit fk
//                                  load); a Bloom hit looks the key up in the
//                                  table; only matching rows load their price and
//                                  discount (late materialisation); exact
//                                  fixed-point sums, 128-bit totals, last block
//                                  writes the result.
// Build-side keys are read densely with the filter columns (one streaming pass).
#include <algorithm>
#include <string>
#include <thread>
#include <utility>

#include "common.cuh"
#include "rows.cuh"
#include "context.cuh"
#include "host_threads.cuh"
#include "mlp.cuh"

namespace bo {

constexpr int kJoinBlock = 512;
constexpr int kBuildBlock = 256;
constexpr int kMinCapLog2 = 10;
// Slots per qualifying build row: a predicted count (presized forms) or the
// exact count (plain form).  Load <= 0.25 at an exact count: measured on B200
// (6M-row probe, 60K keys), a table at load 0.46 probed in 33.0 us, at 0.23 in
// 28.4 us (fewer collisions leave the first slot); sparser tables gain
// little more (26.7 us at 0.06).
constexpr float kPresizeFactor = 4.0f;
constexpr uint64_t kPlainSlotsPerRow = 4;

// Device-resident join state (one per context, in the "join_meta" region).
struct JoinMeta {
  int32_t cap_log2;
  uint32_t done;               // probe ticket counter
  uint32_t overflow;           // presized table too small
  uint32_t pad;
  unsigned long long build_rows;
  unsigned long long distinct;
  unsigned long long acc[6];   // 128-bit totals: matches, sum T, sum rr
  unsigned long long count;    // K7 output
};


// ------------------------------------------------------------ K7 count ----
__global__ void __launch_bounds__(kBuildBlock) join_count_kernel(bo_join_build_cols b, int32_t date_lt, uint32_t seg,
                                                                 unsigned long long* count) {
  uint32_t c = 0;
  const int64_t n = b.n_rows, chunks = n >> 2;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t ch = tid; ch < chunks; ch += stride) {
    const int4 d = ld_stream_v4(b.date + (ch << 2));
    const uint32_t s = ld_stream_u32(b.segment + (ch << 2));
    c += build_qual(d.x, s & 0xffu, date_lt, seg) + build_qual(d.y, (s >> 8) & 0xffu, date_lt, seg) +
         build_qual(d.z, (s >> 16) & 0xffu, date_lt, seg) + build_qual(d.w, s >> 24, date_lt, seg);
  }
  const int64_t t = (chunks << 2) + tid;
  if (t < n) c += build_qual(b.date[t], b.segment[t], date_lt, seg);
  // One atomic per block: per-warp atomics on a single counter serialise in L2.
  __shared__ uint32_t part[kBuildBlock / 32];
  c = warp_sum_u32(c);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tot = 0;
    for (int w = 0; w < kBuildBlock / 32; ++w) tot += part[w];
    if (tot) atomicAdd(count, (unsigned long long)tot);
  }
}

// ------------------------------------------------------------ init -------
// Capacity: host-chosen (exact count) or, when `pred` is given, derived on the
// device from the predicted qualifying-row count: the smallest power of two
// >= kPresizeFactor * pred, clamped to [2^kMinCapLog2, 2^max_log2].  Every block
// computes the same value, so no cross-block handshake is needed.
__device__ __forceinline__ int32_t presize_log2_of(float p, int32_t max_log2) {
  if (!(p >= 0.0f)) p = 0.0f;  // NaN / negative predictions size for the minimum
  const double want = (double)p * kPresizeFactor;
  int32_t cl = kMinCapLog2;
  while (cl < max_log2 && (double)(1ull << cl) < want) ++cl;
  return cl;
}

__device__ __forceinline__ int32_t presize_log2(const float* pred, int32_t host_log2, int32_t max_log2) {
  if (!pred) return host_log2;
  return presize_log2_of(*pred, max_log2);
}

__global__ void join_init_kernel(unsigned long long* slots, uint32_t* bloom, JoinMeta* meta, const float* pred,
                                 int32_t host_log2, int32_t max_log2) {
  pdl_launch_dependents();  // the build kernel may be scheduled now (it waits before touching the table)
  const int32_t cl = presize_log2(pred, host_log2, max_log2);
  const uint64_t cap = 1ull << cl;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  ulonglong2* s2 = reinterpret_cast<ulonglong2*>(slots);
  for (uint64_t i = tid; i < cap / 2; i += stride) s2[i] = make_ulonglong2(kEmptySlot, kEmptySlot);
  uint4* b4 = reinterpret_cast<uint4*>(bloom);
  for (uint64_t i = tid; i < kBloomWords / 4; i += stride) b4[i] = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    meta->cap_log2 = cl;
    meta->done = 0;
    meta->overflow = 0;
    meta->build_rows = 0;
    meta->distinct = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) meta->acc[i] = 0;
  }
}

// The learned form's first kernel: every block evaluates the sizing MLP for
// the query's feature vector (the same instructions on the same inputs, so
// every block derives the same capacity as mlp_predict_counts followed by
// join_init_kernel would), then clears its share of the table and the Bloom
// filter; block 0 resets the join state and records the prediction.  One
// launch instead of two on the query's critical path.
__global__ void __launch_bounds__(kPredThreads) join_learned_init_kernel(const float* __restrict__ params,
                                                                         FeatureVec xv, int F, int O,
                                                                         unsigned long long* slots, uint32_t* bloom,
                                                                         JoinMeta* meta, int32_t max_log2,
                                                                         float* pred_out) {
  __shared__ float y[kMaxO];
  pdl_launch_dependents();  // the build kernel may be scheduled now (it waits before touching the table)
  mlp_predict_block(params, xv, F, O, y);
  const float c = expm1f(y[0]);
  const float pred = c > 0.0f ? c : 0.0f;
  const int32_t cl = presize_log2_of(pred, max_log2);
  const uint64_t cap = 1ull << cl;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  ulonglong2* s2 = reinterpret_cast<ulonglong2*>(slots);
  for (uint64_t i = tid; i < cap / 2; i += stride) s2[i] = make_ulonglong2(kEmptySlot, kEmptySlot);
  uint4* b4 = reinterpret_cast<uint4*>(bloom);
  for (uint64_t i = tid; i < kBloomWords / 4; i += stride) b4[i] = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    meta->cap_log2 = cl;
    meta->done = 0;
    meta->overflow = 0;
    meta->build_rows = 0;
    meta->distinct = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) meta->acc[i] = 0;
    if (pred_out) *pred_out = pred;
  }
}

// ------------------------------------------------------------ K2 build ---

// 16 build rows per thread per step: one 128-bit segment load and two 256-bit
// loads each of dates and keys (the keys are read densely with the filter
// columns: loading only the ~4% qualifying keys afterwards put one more
// dependent DRAM round trip on every warp's path, 2 us per 1.5M-row build on
// B200); the qualifying keys of the whole warp are then compacted into a
// shared-memory queue and inserted by all lanes together.
// kSparseKeys (the streamed forms, whose keys stay in pinned host memory):
// only the qualifying rows' keys are loaded, one 4-byte read over PCIe each,
// instead of the whole key column.
constexpr int kBuildRowsPerThread = 16;

template <bool kSparseKeys>
__global__ void __launch_bounds__(kBuildBlock) join_build_kernel(bo_join_build_cols b, int32_t date_lt, uint32_t seg,
                                                                 unsigned long long* slots, uint32_t* bloom,
                                                                 JoinMeta* meta, uint64_t probe_limit) {
  // Launched right behind the init kernel (programmatic dependent launch):
  // each thread loads and filters its first rows, then waits for the init
  // kernel to finish before it reads the table's size or touches the table.
  pdl_launch_dependents();
  bool waited = false;
  uint64_t mask = 0;
  uint32_t qual = 0, newkeys = 0;
  bool full = false;
  __shared__ uint32_t build_q[kBuildBlock / 32][32 * kBuildRowsPerThread];
  const int lane = threadIdx.x & 31;
  uint32_t* bq = build_q[threadIdx.x >> 5];
  const int64_t n = b.n_rows;
  const int64_t steps = (n + kBuildRowsPerThread - 1) / kBuildRowsPerThread;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  // Every lane of a warp runs the same number of iterations (the bound is
  // rounded up to whole warps) so the warp-wide queue steps stay converged;
  // lanes past the end simply contribute no rows.
  const int64_t steps_w = (steps + 31) & ~int64_t(31);
  for (int64_t st = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; st < steps_w; st += stride) {
    const int64_t r0 = st * kBuildRowsPerThread;
    uint32_t q = 0;
    int32_t keys[kBuildRowsPerThread];
    if (r0 >= n) {
#pragma unroll
      for (int k = 0; k < kBuildRowsPerThread; ++k) keys[k] = 0;
    } else if (r0 + kBuildRowsPerThread <= n) {
      const int4 sg = ld_stream_v4(b.segment + r0);
      const uint32_t sw[4] = {(uint32_t)sg.x, (uint32_t)sg.y, (uint32_t)sg.z, (uint32_t)sg.w};
      const int8v d0 = ld_stream_v8(b.date + r0), d1 = ld_stream_v8(b.date + r0 + 8);
      if constexpr (kSparseKeys) {
#pragma unroll
        for (int k = 0; k < kBuildRowsPerThread; ++k) {
          const int32_t dk = k < 8 ? d0.v[k] : d1.v[k - 8];
          q |= (uint32_t)build_qual(dk, (sw[k >> 2] >> (8 * (k & 3))) & 0xffu, date_lt, seg) << k;
        }
#pragma unroll
        for (int k = 0; k < kBuildRowsPerThread; ++k) keys[k] = ((q >> k) & 1u) ? b.key[r0 + k] : 0;
      } else {
        const int8v k0 = ld_stream_v8(b.key + r0), k1 = ld_stream_v8(b.key + r0 + 8);
#pragma unroll
        for (int k = 0; k < kBuildRowsPerThread; ++k) {
          const int32_t dk = k < 8 ? d0.v[k] : d1.v[k - 8];
          q |= (uint32_t)build_qual(dk, (sw[k >> 2] >> (8 * (k & 3))) & 0xffu, date_lt, seg) << k;
          keys[k] = k < 8 ? k0.v[k] : k1.v[k - 8];
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < kBuildRowsPerThread; ++k) {
        keys[k] = 0;
        if (r0 + k < n && build_qual(b.date[r0 + k], b.segment[r0 + k], date_lt, seg)) {
          q |= 1u << k;
          keys[k] = b.key[r0 + k];
        }
      }
    }
    if (!waited) {
      pdl_wait();
      waited = true;
      // Read-only for this kernel (written by the init kernel): the L1-cached
      // path avoids every warp hitting the same L2 sector.
      mask = (1ull << __ldg(&meta->cap_log2)) - 1;
    }
    qual += __popc(q);
    // Compact the qualifying keys of the whole warp into its queue so the CAS
    // insertions spread over all 32 lanes.
    uint32_t total;
    uint32_t pos = warp_exclusive_scan(__popc(q), total);
    if (total == 0) continue;  // warp-uniform
#pragma unroll
    for (int k = 0; k < kBuildRowsPerThread; ++k)
      if ((q >> k) & 1u) bq[pos++] = (uint32_t)keys[k];
    __syncwarp();
    for (uint32_t i = lane; i < total; i += 32) join_insert(slots, bloom, mask, (int32_t)bq[i], newkeys, full, probe_limit);
    __syncwarp();
  }
  if (!waited) pdl_wait();  // threads without rows: before the counters below
  // Block-level totals, then one atomic per counter per block.
  __shared__ uint32_t part[3][kBuildBlock / 32];
  const uint32_t wq = warp_sum_u32(qual), wn = warp_sum_u32(newkeys);
  const unsigned any_full = __any_sync(0xffffffffu, full);
  if ((threadIdx.x & 31) == 0) {
    part[0][threadIdx.x >> 5] = wq;
    part[1][threadIdx.x >> 5] = wn;
    part[2][threadIdx.x >> 5] = any_full;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tq = 0, tn = 0, tf = 0;
    for (int w = 0; w < kBuildBlock / 32; ++w) {
      tq += part[0][w];
      tn += part[1][w];
      tf |= part[2][w];
    }
    if (tq) atomicAdd(&meta->build_rows, (unsigned long long)tq);
    if (tn) {
      const unsigned long long before = atomicAdd(&meta->distinct, (unsigned long long)tn);
      // A presized table is "too small" once it is more than 7/8 occupied.
      if (before + tn > (mask + 1) - ((mask + 1) >> 3)) atomicOr(&meta->overflow, 1u);
    }
    if (tf) atomicOr(&meta->overflow, 1u);
  }
}

// ------------------------------------------------------------ K3 probe ---

// Warp-centric probe.  A warp owns 256 consecutive probe rows per step (8 per
// lane, one 256-bit fk load).  Every lane hashes its rows and tests the Bloom
// filter in shared memory without branching; the hits (about 9% of rows) are
// compacted into a per-warp shared-memory queue (ballot-free: a warp prefix sum
// of per-lane hit counts gives each lane its slot range), and then all 32 lanes
// resolve queue entries together -- table lookups and the price / discount
// loads of matches are issued by many lanes at once instead of one row at a
// time.  The queue holds a whole step.  (Steps of 512 rows resolved in two
// halves took 32 us per 6M-row launch on B200, steps of 256 rows 27.5 us:
// more, shorter dependent chains in flight per SM.)
constexpr int kProbeWarps = kJoinBlock / 32;
constexpr int kRowsPerLane = 8;
constexpr int kRowsPerWarpStep = 32 * kRowsPerLane;
constexpr int kQueue = 32 * kRowsPerLane;
constexpr int kJoinResolveR = 2;  // candidates per lane per resolve round

// Match list of the host-gather form: instead of reading price / discount
// over PCIe, the probe appends each matching row (relative to the launch's
// first row) to pinned host memory and its build-side multiplicity to device
// memory; the host gathers the payload of exactly those rows.
struct EmitOut {
  uint32_t* rows = nullptr;        // device view of mapped host memory
  uint32_t* mult = nullptr;        // device memory, same index as rows
  uint32_t* counter = nullptr;     // device: entries appended (zeroed again by the last block)
  uint32_t* count_host = nullptr;  // device view of mapped host memory: the launch's entry count
  uint32_t capacity = 0;
};

// probe_resolve's lookups, then warp-aggregated appends of the matches (one
// atomic per warp and round) in place of the payload loads.
template <int R>
__device__ __forceinline__ void probe_emit(const int32_t* qf, const uint16_t* qo, uint32_t total, int64_t base,
                                           const unsigned long long* slots, uint64_t mask, uint64_t limit,
                                           const EmitOut& eo, ProbeAcc& acc) {
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
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
    unsigned long long mult[R];
    uint32_t bal[R], n = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      mult[r] = 0;
      if (v[r] != kEmptySlot) {
        if ((uint32_t)(v[r] >> 32) == (uint32_t)key[r])
          mult[r] = v[r] & 0xffffffffull;
        else
          mult[r] = probe_slow<false>(slots, mask, idx[r], (uint32_t)key[r], limit);
      }
      bal[r] = __ballot_sync(0xffffffffu, mult[r] != 0);
      n += __popc(bal[r]);
    }
    if (n == 0) continue;  // warp-uniform
    uint32_t pos = 0;
    if (lane == 0) pos = atomicAdd(eo.counter, n);
    pos = __shfl_sync(0xffffffffu, pos, 0);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (mult[r]) {
        const uint32_t at = pos + __popc(bal[r] & lt);
        if (at < eo.capacity) {
          eo.rows[at] = (uint32_t)row[r];
          eo.mult[at] = (uint32_t)mult[r];
          acc.cnt += mult[r];
        } else {
          acc.bad |= kErrOutputOverflow;
        }
      }
      pos += __popc(bal[r]);
    }
  }
}

template <bool kEmit>
__global__ void __launch_bounds__(kJoinBlock, 2) join_probe_kernel(bo_join_probe_cols p,
                                                                const unsigned long long* slots,
                                                                const uint32_t* bloom_g, JoinMeta* meta,
                                                                bo_join_result* out, int32_t mode, uint64_t probe_limit,
                                                                uint32_t* err, EmitOut eo) {
  extern __shared__ __align__(128) uint32_t bloom_s[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ unsigned __int128 red[kJoinBlock + 32];
  __shared__ int32_t q_fk[kProbeWarps][kQueue];
  __shared__ uint16_t q_off[kProbeWarps][kQueue];
  pdl_wait();  // launched behind the build kernel: its table and Bloom filter must be complete
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_arrive_expect_tx(&bar, kBloomBytes);
    bulk_copy_g2s(bloom_s, bloom_g, kBloomBytes, &bar);
  }
  __syncthreads();
  // On a (never expected) timeout the filter is simply not used: every row then
  // probes the table directly, which gives the same answer.
  const bool use_bloom = mbar_wait_bounded(&bar, 0, kWaitLimitNs);
  ProbeAcc acc;
  if (!use_bloom) acc.bad |= kErrSpinTimeout;
  __shared__ uint32_t all_ones;
  if (threadIdx.x == 0) all_ones = 0xffffffffu;
  __syncthreads();
  const uint32_t* bl = use_bloom ? bloom_s : &all_ones;
  const uint32_t wmask = use_bloom ? (kBloomWords - 1u) : 0u;

  const int32_t cl = __ldg(&meta->cap_log2);
  const uint64_t mask = (1ull << cl) - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int32_t* qf = q_fk[warp];
  uint16_t* qo = q_off[warp];
  const int64_t n = p.n_rows;
  const int64_t steps = (n + kRowsPerWarpStep - 1) / kRowsPerWarpStep;
  const int64_t nwarps = (int64_t)gridDim.x * kProbeWarps;
  for (int64_t st = (int64_t)blockIdx.x * kProbeWarps + warp; st < steps; st += nwarps) {
    const int64_t base = st * kRowsPerWarpStep;
    const int64_t r0 = base + lane * kRowsPerLane;
    int32_t fk[kRowsPerLane];
    uint32_t valid = 0xffu;
    if (r0 + kRowsPerLane <= n) {
      const int8v f0 = ld_first_v8(p.fk + r0);  // the table and payload lookups keep L2
#pragma unroll
      for (int k = 0; k < kRowsPerLane; ++k) fk[k] = f0.v[k];
    } else {
      valid = 0;
#pragma unroll
      for (int k = 0; k < kRowsPerLane; ++k) {
        fk[k] = 0;
        if (r0 + k < n) {
          fk[k] = p.fk[r0 + k];
          valid |= 1u << k;
        }
      }
    }
    // Branch-free Bloom test (without the filter every word reads as all ones).
    uint32_t hit = 0;
#pragma unroll
    for (int k = kRowsPerLane - 1; k >= 0; --k) hit = (hit << 1) | bloom_test(bl, wmask, (uint32_t)fk[k]);
    hit &= valid;
    uint32_t total;
    uint32_t pos = warp_exclusive_scan(__popc(hit), total);
#pragma unroll
    for (int k = 0; k < kRowsPerLane; ++k) {
      if ((hit >> k) & 1u) {
        qf[pos] = fk[k];
        qo[pos] = (uint16_t)(lane * kRowsPerLane + k);
        ++pos;
      }
    }
    __syncwarp();
    if constexpr (kEmit)
      probe_emit<kJoinResolveR>(qf, qo, total, base, slots, mask, probe_limit, eo, acc);
    else
      probe_resolve<kJoinResolveR, false>(qf, qo, total, base, slots, mask, probe_limit, p.price, p.discount, acc);
    __syncwarp();
  }
  if (!use_bloom) {
    // The bulk copy may still be in flight: wait for it (bounded) before exit.
    mbar_wait_bounded(&bar, 0, kWaitLimitNs);
  }
  if (acc.bad) raise_error(err, acc.bad);
  const unsigned long long cnt = acc.cnt, rsum = acc.rsum;
  const unsigned __int128 tsum = acc.tsum;

  const unsigned __int128 bc = block_sum_u128(cnt, red);
  const unsigned __int128 bt = block_sum_u128(tsum, red);
  const unsigned __int128 br = block_sum_u128(rsum, red);
  if (threadIdx.x == 0) {
    if (bc) atomic_add_i128(&meta->acc[0], (__int128)bc);
    if (bt) atomic_add_i128(&meta->acc[2], (__int128)bt);
    if (br) atomic_add_i128(&meta->acc[4], (__int128)br);
  }
  if (last_block(&meta->done)) {
    if (threadIdx.x == 0) {
      uint32_t fbad = 0;
      const __int128 m = load_i128(&meta->acc[0]), t = load_i128(&meta->acc[2]), rr = load_i128(&meta->acc[4]);
      bo_join_result res;
      res.build_rows = (int64_t)__ldcg(&meta->build_rows);
      res.distinct_keys = (int64_t)__ldcg(&meta->distinct);
      res.match_count = narrow_i64(m, fbad);
      res.sum_trunc = to_bo_i128(t);
      res.sum_exact = to_bo_i128(t * 100 + rr);
      res.capacity_log2 = cl;
      res.overflowed = (int32_t)__ldcg(&meta->overflow);
      res.reruns = 0;
      res.mode = mode;
      *out = res;
#pragma unroll
      for (int i = 0; i < 6; ++i) meta->acc[i] = 0;
      meta->done = 0;
      if constexpr (kEmit) {
        const uint32_t entries = atomicExch(eo.counter, 0u);
        *reinterpret_cast<volatile uint32_t*>(eo.count_host) = entries < eo.capacity ? entries : eo.capacity;
      }
      if (fbad) raise_error(err, fbad);
    }
  }
}

// Host-gather form, second half: the payload of a probe launch's matches,
// gathered on the host into (price, discount) records and copied in, summed
// with the multiplicities the probe kept; the last block adds the totals to
// that launch's partial result (whose match count the probe wrote).
struct GatherAcc {
  unsigned long long acc[4];  // 128-bit totals: sum T, sum rr
  uint32_t done;
  uint32_t pad;
};

constexpr int kGatherBlock = 256;

__global__ void __launch_bounds__(kGatherBlock) join_gather_sum_kernel(const uint2* __restrict__ rec,
                                                                       const uint32_t* __restrict__ mult, int64_t n,
                                                                       GatherAcc* ga, bo_join_result* part,
                                                                       uint32_t* err) {
  __shared__ unsigned __int128 red[kGatherBlock + 32];
  ProbeAcc a;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint2 r = __ldcs(rec + i);
    accumulate_match((uint64_t)r.x, (uint64_t)r.y, __ldcs(mult + i), a);
  }
  if (a.bad) raise_error(err, a.bad);
  const unsigned __int128 bt = block_sum_u128(a.tsum, red);
  const unsigned __int128 br = block_sum_u128(a.rsum, red);
  if (threadIdx.x == 0) {
    if (bt) atomic_add_i128(&ga->acc[0], (__int128)bt);
    if (br) atomic_add_i128(&ga->acc[2], (__int128)br);
  }
  if (last_block(&ga->done) && threadIdx.x == 0) {
    const __int128 t = load_i128(&ga->acc[0]), rr = load_i128(&ga->acc[2]);
    part->sum_trunc = to_bo_i128(t);
    part->sum_exact = to_bo_i128(t * 100 + rr);
#pragma unroll
    for (int i = 0; i < 4; ++i) ga->acc[i] = 0;
    ga->done = 0;
  }
}

// ------------------------------------------------------------------ host ---
namespace {

struct JoinWs {
  unsigned long long* slots;
  uint32_t* bloom;
  JoinMeta* meta;
  float* pred;
  int32_t max_log2;
};

int ceil_log2(uint64_t v) {
  int l = 0;
  while ((1ull << l) < v) ++l;
  return l;
}

int join_workspace(bo_ctx* ctx, int64_t n_build, JoinWs* ws) {
  // The table never needs more than 2 slots per build row (exact sizing uses
  // 2x the exact count; predictions are clamped to this bound).
  const int32_t max_log2 = std::max(kMinCapLog2, ceil_log2((uint64_t)std::max<int64_t>(n_build, 1) * 2));
  void* p = nullptr;
  int rc = region(ctx, "join_slots", sizeof(unsigned long long) << max_log2, &p);
  if (rc) return rc;
  ws->slots = static_cast<unsigned long long*>(p);
  if ((rc = region(ctx, "join_bloom", kBloomBytes, &p))) return rc;
  ws->bloom = static_cast<uint32_t*>(p);
  if ((rc = region(ctx, "join_meta", sizeof(JoinMeta) + 64, &p))) return rc;
  ws->meta = static_cast<JoinMeta*>(p);
  ws->pred = reinterpret_cast<float*>(static_cast<char*>(p) + sizeof(JoinMeta));
  ws->max_log2 = max_log2;
  return BO_OK;
}

int check_join(bo_ctx* ctx, const bo_join_build_cols* b, const bo_join_probe_cols* p, const bo_join_params* prm) {
  if (!b || !p || !prm) return set_error(ctx, BO_ERR_INVALID, "join: null argument");
  if (b->n_rows < 0 || p->n_rows < 0) return set_error(ctx, BO_ERR_INVALID, "join: negative row count");
  if (b->n_rows > 0x7fffffffll) return set_error(ctx, BO_ERR_INVALID, "join: build side above 2^31 rows");
  if (b->n_rows > 0) {
    const void* bp[] = {b->key, b->date, b->segment};
    for (const void* x : bp)
      if (!x || !aligned32(x)) return set_error(ctx, BO_ERR_INVALID, "join: build column null or not 32-byte aligned");
  }
  if (p->n_rows > 0) {
    const void* pp[] = {p->fk, p->price, p->discount};
    for (const void* x : pp)
      if (!x || !aligned32(x)) return set_error(ctx, BO_ERR_INVALID, "join: probe column null or not 32-byte aligned");
  }
  if (prm->segment_eq < 0 || prm->segment_eq > 255)
    return set_error(ctx, BO_ERR_INVALID, "join: segment_eq %d outside uint8", prm->segment_eq);
  return BO_OK;
}

int grid_for(bo_ctx* ctx, const void* k, int block, size_t smem, int64_t work_items) {
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(k, block, smem);
  int64_t need = (work_items + block - 1) / block;
  int64_t g = std::min<int64_t>(resident, std::max<int64_t>(need, 1));
  return (int)std::max<int64_t>(g, 1);
}

// Launches a kernel that may start while the previous kernel on the stream
// still runs (programmatic dependent launch); the kernel itself waits
// (pdl_wait) before it reads that kernel's output.
template <typename... KArgs, typename... Args>
cudaError_t launch_dependent(void (*k)(KArgs...), int grid, int block, size_t smem, cudaStream_t st,
                             Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

// Probe launch; a match list (eo.rows set) selects the host-gather form.
int launch_probe(bo_ctx* ctx, const bo_join_probe_cols& p, const JoinWs& ws, bo_join_result* out, int32_t mode,
                 uint64_t probe_limit, bool dependent = false, const EmitOut& eo = EmitOut()) {
  const bool emit = eo.rows != nullptr;
  auto* kfn = emit ? &join_probe_kernel<true> : &join_probe_kernel<false>;
  const void* k = reinterpret_cast<const void*>(kfn);
  static bool ready[2] = {false, false};
  if (!ready[emit]) {
    BO_CUDA(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBloomBytes));
    ready[emit] = true;
  }
  // Enough blocks to fill the GPU, but each thread should see a few 8-row
  // chunks so the per-block Bloom-filter copy is amortised.
  const int grid = grid_for(ctx, k, kJoinBlock, kBloomBytes, (p.n_rows + kRowsPerLane - 1) / kRowsPerLane);
  if (dependent)
    BO_CUDA(ctx, launch_dependent(kfn, grid, kJoinBlock, kBloomBytes, ctx->stream, p,
                                  (const unsigned long long*)ws.slots, (const uint32_t*)ws.bloom, ws.meta, out, mode,
                                  probe_limit, ctx->d_err, eo));
  else
    kfn<<<grid, kJoinBlock, kBloomBytes, ctx->stream>>>(p, ws.slots, ws.bloom, ws.meta, out, mode, probe_limit,
                                                        ctx->d_err, eo);
  return after_launch(ctx, "join_probe_kernel");
}

// init + build + probe, asynchronous.
int join_run(bo_ctx* ctx, const bo_join_build_cols& b, const bo_join_probe_cols& p, const bo_join_params& prm,
             const JoinWs& ws, const float* pred, int32_t host_log2, bo_join_result* out, int32_t mode) {
  const void* ki = reinterpret_cast<const void*>(&join_init_kernel);
  const int gi = grid_for(ctx, ki, 256, 0, (int64_t)1 << std::min(ws.max_log2, 24));
  join_init_kernel<<<gi, 256, 0, ctx->stream>>>(ws.slots, ws.bloom, ws.meta, pred, host_log2, ws.max_log2);
  int rc = after_launch(ctx, "join_init_kernel");
  if (rc) return rc;
  const void* kb = reinterpret_cast<const void*>(&join_build_kernel<false>);
  const int gb = grid_for(ctx, kb, kBuildBlock, 0, (b.n_rows + kBuildRowsPerThread - 1) / kBuildRowsPerThread);
  // Exact-size tables (mode 0) probe without a bound; presized ones fail fast.
  const uint64_t limit = mode == 0 ? ~0ull : kPresizedProbeLimit;
  BO_CUDA(ctx, launch_dependent(&join_build_kernel<false>, gb, kBuildBlock, 0, ctx->stream, b, prm.date_lt,
                                (uint32_t)prm.segment_eq, ws.slots, ws.bloom, ws.meta, limit));
  if ((rc = after_launch(ctx, "join_build_kernel"))) return rc;
  return launch_probe(ctx, p, ws, out, mode, limit, true);
}

int finish_join(bo_ctx* ctx, bo_join_result* host, const bo_join_result* dev) {
  BO_CUDA(ctx, cudaMemcpyAsync(host, dev, sizeof(bo_join_result), cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  int rc = consume_device_errors(ctx, &bits);
  if (rc) return rc;
  return device_error_status(ctx, bits, "join");
}

int join_plain_impl(bo_ctx* ctx, const bo_join_build_cols& b, const bo_join_probe_cols& p, const bo_join_params& prm,
                    bo_join_result* out_host, int32_t reruns) {
  JoinWs ws;
  int rc = join_workspace(ctx, b.n_rows, &ws);
  if (rc) return rc;
  // K7: exact count, then one host round trip to size the table.
  BO_CUDA(ctx, cudaMemsetAsync(&ws.meta->count, 0, sizeof(unsigned long long), ctx->stream));
  const void* kc = reinterpret_cast<const void*>(&join_count_kernel);
  const int gc = grid_for(ctx, kc, kBuildBlock, 0, (b.n_rows + 3) / 4);
  join_count_kernel<<<gc, kBuildBlock, 0, ctx->stream>>>(b, prm.date_lt, (uint32_t)prm.segment_eq, &ws.meta->count);
  if ((rc = after_launch(ctx, "join_count_kernel"))) return rc;
  unsigned long long count = 0;
  BO_CUDA(ctx, cudaMemcpyAsync(&count, &ws.meta->count, sizeof(count), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const int32_t cl = std::min(ws.max_log2, std::max(kMinCapLog2, ceil_log2(std::max<uint64_t>(count, 1) * kPlainSlotsPerRow)));
  void* dout = nullptr;
  if ((rc = region(ctx, "join_out", sizeof(bo_join_result), &dout))) return rc;
  bo_join_result* d = static_cast<bo_join_result*>(dout);
  if ((rc = join_run(ctx, b, p, prm, ws, nullptr, cl, d, 0))) return rc;
  if ((rc = finish_join(ctx, out_host, d))) return rc;
  out_host->reruns = reruns;
  if (out_host->overflowed)  // cannot happen with exact sizing; report rather than loop
    return set_error(ctx, BO_ERR_OVERFLOW, "join: exact-size table overflowed");
  return BO_OK;
}

// ------------------------------------------------------ streamed join ---
// Inputs in pinned host memory: the dense columns (build date and segment,
// probe fk) are copied on the context's copy stream, fk in chunks; the kernels
// read the build keys of qualifying rows and the price / discount of matching
// rows in place.  Two buffer sets alternate so that a query's copies overlap
// the previous query's kernels; a set is reused only after the compute stream
// has finished with it (its "done" event).
constexpr int64_t kStreamChunkRows = 1 << 20;  // probe rows per copy / probe step

__global__ void join_combine_kernel(const bo_join_result* __restrict__ part, int64_t n, bo_join_result* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  bo_join_result r = part[0];
  __int128 se = 0, st = 0;
  int64_t mc = 0;
  int32_t of = 0;
  for (int64_t i = 0; i < n; ++i) {
    se += ((__int128)part[i].sum_exact.hi << 64) | part[i].sum_exact.lo;
    st += ((__int128)part[i].sum_trunc.hi << 64) | part[i].sum_trunc.lo;
    mc += part[i].match_count;
    of |= part[i].overflowed;
  }
  r.match_count = mc;
  r.sum_exact = to_bo_i128(se);
  r.sum_trunc = to_bo_i128(st);
  r.overflowed = of;
  r.reruns = 0;
  *out = r;
}

// Device pointer of a pinned (mapped) host buffer, or null if it is not one.
const void* mapped_device_pointer(const void* host) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, host) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
  return a.devicePointer;
}

struct StreamIn {
  const int32_t* key = nullptr;    // device views of pinned host columns
  const int64_t* price = nullptr;
  const int64_t* disc = nullptr;
  int64_t chunks = 1;
};

int stream_check(bo_ctx* ctx, const bo_join_build_cols* bh, const bo_join_probe_cols* ph, const bo_join_params* prm,
                 StreamIn* in) {
  if (!bh || !ph || !prm) return set_error(ctx, BO_ERR_INVALID, "join_stream: null argument");
  if (bh->n_rows < 0 || ph->n_rows < 0 || bh->n_rows > 0x7fffffffll)
    return set_error(ctx, BO_ERR_INVALID, "join_stream: row counts");
  if (prm->segment_eq < 0 || prm->segment_eq > 255)
    return set_error(ctx, BO_ERR_INVALID, "join_stream: segment_eq %d outside uint8", prm->segment_eq);
  if (bh->n_rows > 0) {
    in->key = static_cast<const int32_t*>(mapped_device_pointer(bh->key));
    if (!in->key || !mapped_device_pointer(bh->date) || !mapped_device_pointer(bh->segment))
      return set_error(ctx, BO_ERR_INVALID, "join_stream: build columns must be pinned host memory");
  }
  if (ph->n_rows > 0) {
    in->price = static_cast<const int64_t*>(mapped_device_pointer(ph->price));
    in->disc = static_cast<const int64_t*>(mapped_device_pointer(ph->discount));
    if (!in->price || !in->disc || !mapped_device_pointer(ph->fk))
      return set_error(ctx, BO_ERR_INVALID, "join_stream: probe columns must be pinned host memory");
  }
  in->chunks = std::max<int64_t>(1, (ph->n_rows + kStreamChunkRows - 1) / kStreamChunkRows);
  return BO_OK;
}

struct StreamSet {
  int32_t* date;
  uint8_t* seg;
  int32_t* fk;
  bo_join_result* part;
  bo_join_result* combined;
};

size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

int stream_set(bo_ctx* ctx, int64_t nb, int64_t np, int64_t chunks, int set, StreamSet* s) {
  const size_t b_date = al256(4 * (size_t)nb), b_seg = al256((size_t)nb), b_fk = al256(4 * (size_t)np);
  const size_t b_part = al256(sizeof(bo_join_result) * (size_t)(chunks + 1));
  const size_t per = b_date + b_seg + b_fk + b_part;
  void* base = nullptr;
  int rc = region(ctx, "join_stream", 2 * per, &base);
  if (rc) return rc;
  char* p = static_cast<char*>(base) + (size_t)set * per;
  s->date = reinterpret_cast<int32_t*>(p);
  s->seg = reinterpret_cast<uint8_t*>(p + b_date);
  s->fk = reinterpret_cast<int32_t*>(p + b_date + b_seg);
  s->part = reinterpret_cast<bo_join_result*>(p + b_date + b_seg + b_fk);
  s->combined = s->part + chunks;
  return BO_OK;
}

// Events: [0], [1] "set done"; [2] build columns copied; [3 + c] probe chunk c copied.
int stream_events(bo_ctx* ctx, int64_t chunks) {
  while (ctx->events.size() < (size_t)(chunks + 3)) {
    cudaEvent_t e;
    BO_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->events.push_back(e);
  }
  return BO_OK;
}

int stream_copies(bo_ctx* ctx, const bo_join_build_cols* bh, const bo_join_probe_cols* ph, const StreamIn& in,
                  const StreamSet& s, int set) {
  if (!ctx->copy_stream) BO_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  cudaStream_t cs = ctx->copy_stream;
  cudaEvent_t* ev = ctx->events.data();
  BO_CUDA(ctx, cudaStreamWaitEvent(cs, ev[set], 0));  // the set's previous query has finished with it
  const int64_t nb = bh->n_rows, np = ph->n_rows;
  if (nb > 0) {
    BO_CUDA(ctx, cudaMemcpyAsync(s.date, bh->date, 4 * (size_t)nb, cudaMemcpyHostToDevice, cs));
    BO_CUDA(ctx, cudaMemcpyAsync(s.seg, bh->segment, (size_t)nb, cudaMemcpyHostToDevice, cs));
  }
  BO_CUDA(ctx, cudaEventRecord(ev[2], cs));
  for (int64_t c = 0; c < in.chunks; ++c) {
    const int64_t lo = c * kStreamChunkRows, n = std::min(np - lo, kStreamChunkRows);
    if (n > 0) BO_CUDA(ctx, cudaMemcpyAsync(s.fk + lo, ph->fk + lo, 4 * (size_t)n, cudaMemcpyHostToDevice, cs));
    BO_CUDA(ctx, cudaEventRecord(ev[3 + c], cs));
  }
  return BO_OK;
}

// init + build + chunked probe + combine on the compute stream; the caller
// made the compute stream wait for ev[2] already when it sized the table from
// an exact count (pred == nullptr).
int stream_compute(bo_ctx* ctx, const bo_join_build_cols* bh, const bo_join_probe_cols* ph, const bo_join_params* prm,
                   const float* pred, int32_t host_log2, const JoinWs& ws, const StreamIn& in, const StreamSet& s,
                   int set) {
  cudaEvent_t* ev = ctx->events.data();
  BO_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ev[2], 0));
  const int64_t nb = bh->n_rows, np = ph->n_rows;
  const int32_t mode = pred ? 1 : 0;
  const uint64_t limit = mode == 0 ? ~0ull : kPresizedProbeLimit;
  const bo_join_build_cols b = {in.key, s.date, s.seg, nb};
  const void* ki = reinterpret_cast<const void*>(&join_init_kernel);
  join_init_kernel<<<grid_for(ctx, ki, 256, 0, (int64_t)1 << std::min(ws.max_log2, 24)), 256, 0, ctx->stream>>>(
      ws.slots, ws.bloom, ws.meta, pred, host_log2, ws.max_log2);
  int rc = after_launch(ctx, "join_init_kernel");
  if (rc) return rc;
  const void* kb = reinterpret_cast<const void*>(&join_build_kernel<true>);
  join_build_kernel<true><<<grid_for(ctx, kb, kBuildBlock, 0, (nb + kBuildRowsPerThread - 1) / kBuildRowsPerThread),
                      kBuildBlock, 0, ctx->stream>>>(b, prm->date_lt, (uint32_t)prm->segment_eq, ws.slots, ws.bloom,
                                                     ws.meta, limit);
  if ((rc = after_launch(ctx, "join_build_kernel"))) return rc;
  for (int64_t c = 0; c < in.chunks; ++c) {
    const int64_t lo = c * kStreamChunkRows, n = std::max<int64_t>(0, std::min(np - lo, kStreamChunkRows));
    BO_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ev[3 + c], 0));
    const bo_join_probe_cols pc = {s.fk + lo, in.price ? in.price + lo : nullptr, in.disc ? in.disc + lo : nullptr, n};
    if ((rc = launch_probe(ctx, pc, ws, s.part + c, mode, limit))) return rc;
  }
  join_combine_kernel<<<1, 32, 0, ctx->stream>>>(s.part, in.chunks, s.combined);
  if ((rc = after_launch(ctx, "join_combine_kernel"))) return rc;
  BO_CUDA(ctx, cudaEventRecord(ev[set], ctx->stream));
  return BO_OK;
}

// ---------------------------------------- streamed join, host gather ---
// Of a probe row's 16 payload bytes (price, discount) only the matching rows'
// are needed, a few percent.  Read in place over PCIe each match costs two
// small read requests, and the link serves those about one round trip at a
// time (0.6 ms for 240K matches on B200 behind PCIe 5).  In this form the
// probe lists the matching rows in pinned host memory instead; host threads
// gather those rows' payload into contiguous (price, discount) records while
// later chunks are still being copied and probed, and one bulk copy per chunk
// brings the records to a summing kernel.  The gather's device work runs on
// its own stream, enqueued by the context's HostQueue thread, so the caller
// never waits for it; bo_synchronize (or any synchronous call) drains it.
constexpr int kGatherRing = 4;  // staging buffers of gathered records in flight

}  // namespace

struct GatherSet {
  uint32_t* rows_h = nullptr;       // pinned, mapped: chunk c's match rows from c * kStreamChunkRows
  uint32_t* rows_d = nullptr;       // device view of rows_h
  uint32_t* count_h = nullptr;      // pinned, mapped: entries per chunk
  uint32_t* count_d = nullptr;      // device view of count_h
  uint32_t* mult = nullptr;         // device: multiplicities, laid out as rows_h
  uint32_t* counter = nullptr;      // device: per-chunk append counters
  bo_join_result* res_h = nullptr;  // pinned result slot of the synchronous form
  std::vector<cudaEvent_t> probed;  // chunk c's probe has finished
  uint64_t ticket = 0;              // queue task of the set's latest query
};

struct GatherState {
  GatherState(int device, int threads) : pool(threads), queue([device] { cudaSetDevice(device); }) {}
  HostPool pool;    // declared before the queue: the queue's tasks use it
  HostQueue queue;
  cudaStream_t stream = nullptr;
  GatherSet set[2];
  int64_t rows_cap = 0, chunk_cap = 0;  // per set
  uint2* rec_h[kGatherRing] = {};       // pinned staging, kStreamChunkRows records each
  cudaEvent_t rec_ev[kGatherRing] = {};  // the copy out of rec_h[i] has finished
  bool rec_busy[kGatherRing] = {};
  int next_rec = 0;
  uint2* rec_d = nullptr;  // kGatherRing x kStreamChunkRows records
  GatherAcc* acc = nullptr;
};

namespace {

int auto_gather_threads() {
  const unsigned hc = std::thread::hardware_concurrency();
  return (int)std::min(8u, std::max(1u, hc / 2));
}

void free_gather_sets(GatherState* g) {
  for (GatherSet& st : g->set) {
    if (st.rows_h) cudaFreeHost(st.rows_h);
    if (st.count_h) cudaFreeHost(st.count_h);
    if (st.res_h) cudaFreeHost(st.res_h);
    if (st.mult) cudaFree(st.mult);
    if (st.counter) cudaFree(st.counter);
    for (cudaEvent_t e : st.probed) cudaEventDestroy(e);
    st = GatherSet();
  }
  g->rows_cap = g->chunk_cap = 0;
}

void free_gather(GatherState* g) {
  free_gather_sets(g);
  for (int i = 0; i < kGatherRing; ++i) {
    if (g->rec_h[i]) cudaFreeHost(g->rec_h[i]);
    if (g->rec_ev[i]) cudaEventDestroy(g->rec_ev[i]);
  }
  if (g->rec_d) cudaFree(g->rec_d);
  if (g->acc) cudaFree(g->acc);
  if (g->stream) cudaStreamDestroy(g->stream);
}

// The context's gather state (created on first use), or null in *out when the
// context reads the payload in place (no gather threads).
int gather_state(bo_ctx* ctx, GatherState** out) {
  *out = nullptr;
  const int threads = ctx->gather_threads < 0 ? auto_gather_threads() : ctx->gather_threads;
  if (threads == 0) return BO_OK;
  if (!ctx->gather) {
    auto* g = new GatherState(ctx->device, threads);
    auto init = [&]() -> int {
      BO_CUDA(ctx, cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
      for (int i = 0; i < kGatherRing; ++i) {
        BO_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void**>(&g->rec_h[i]), sizeof(uint2) * kStreamChunkRows,
                                   cudaHostAllocDefault));
        BO_CUDA(ctx, cudaEventCreateWithFlags(&g->rec_ev[i], cudaEventDisableTiming));
      }
      BO_CUDA(ctx, cudaMalloc(&g->rec_d, sizeof(uint2) * kStreamChunkRows * kGatherRing));
      BO_CUDA(ctx, cudaMalloc(&g->acc, sizeof(GatherAcc)));
      BO_CUDA(ctx, cudaMemset(g->acc, 0, sizeof(GatherAcc)));
      return BO_OK;
    };
    if (int rc = init()) {
      free_gather(g);
      delete g;
      return rc;
    }
    ctx->gather = g;
  }
  *out = ctx->gather;
  return BO_OK;
}

// Per-set buffers for `np` probe rows in `chunks` chunks; growing them first
// drains every queued gather (their tasks hold the old buffers).
int gather_reserve(bo_ctx* ctx, GatherState* g, int64_t np, int64_t chunks) {
  const int64_t rows = std::max<int64_t>(np, 1);
  if (rows <= g->rows_cap && chunks <= g->chunk_cap) return BO_OK;
  if (int rc = drain_host_work(ctx)) return rc;
  free_gather_sets(g);
  for (GatherSet& st : g->set) {
    BO_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void**>(&st.rows_h), sizeof(uint32_t) * rows, cudaHostAllocMapped));
    BO_CUDA(ctx, cudaHostGetDevicePointer(reinterpret_cast<void**>(&st.rows_d), st.rows_h, 0));
    BO_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void**>(&st.count_h), sizeof(uint32_t) * chunks, cudaHostAllocMapped));
    BO_CUDA(ctx, cudaHostGetDevicePointer(reinterpret_cast<void**>(&st.count_d), st.count_h, 0));
    BO_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void**>(&st.res_h), sizeof(bo_join_result), cudaHostAllocDefault));
    BO_CUDA(ctx, cudaMalloc(&st.mult, sizeof(uint32_t) * rows));
    BO_CUDA(ctx, cudaMalloc(&st.counter, sizeof(uint32_t) * chunks));
    BO_CUDA(ctx, cudaMemset(st.counter, 0, sizeof(uint32_t) * chunks));
    st.probed.resize(chunks);
    for (cudaEvent_t& e : st.probed) BO_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  g->rows_cap = rows;
  g->chunk_cap = chunks;
  return BO_OK;
}

// (price, discount) of the listed rows [b, e) into records; the rows of one
// warp's appends are close together, so prefetching a few entries ahead keeps
// several cache misses in flight per thread.
void gather_rows(const uint32_t* rows, const int64_t* price, const int64_t* disc, uint2* out, int64_t b,
                 int64_t e) {
  constexpr int64_t kAhead = 16;
  for (int64_t i = b; i < e; ++i) {
    if (i + kAhead < e) {
      const uint32_t ra = rows[i + kAhead];
      __builtin_prefetch(price + ra);
      __builtin_prefetch(disc + ra);
    }
    const uint32_t r = rows[i];
    const int64_t pv = price[r], dv = disc[r];
    // 4 + 4 bytes: the exact-arithmetic contract (0 <= price < 2^31, 0 <=
    // discount <= 100) fits; a value outside it becomes a price the summing
    // kernel rejects (a data error, as in the in-place form).
    const bool ok = pv >= 0 && pv < 0x80000000ll && dv >= 0 && dv <= 100;
    out[i] = make_uint2(ok ? (uint32_t)pv : 0xffffffffu, ok ? (uint32_t)dv : 0u);
  }
}

// init + build + chunked listing probe on the compute stream, then the
// gather task: per chunk, wait for its probe, gather, copy the records in and
// sum them on the gather stream; combine, and copy the result to `dst`
// (pinned host memory).
int stream_compute_gather(bo_ctx* ctx, GatherState* g, const bo_join_build_cols* bh, const bo_join_probe_cols* ph,
                          const bo_join_params* prm, const float* pred, int32_t host_log2, const JoinWs& ws,
                          const StreamIn& in, const StreamSet& s, int set, bo_join_result* dst) {
  cudaEvent_t* ev = ctx->events.data();
  GatherSet& gs = g->set[set];
  BO_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ev[2], 0));
  const int64_t nb = bh->n_rows, np = ph->n_rows;
  const int32_t mode = pred ? 1 : 0;
  const uint64_t limit = mode == 0 ? ~0ull : kPresizedProbeLimit;
  const bo_join_build_cols b = {in.key, s.date, s.seg, nb};
  const void* ki = reinterpret_cast<const void*>(&join_init_kernel);
  join_init_kernel<<<grid_for(ctx, ki, 256, 0, (int64_t)1 << std::min(ws.max_log2, 24)), 256, 0, ctx->stream>>>(
      ws.slots, ws.bloom, ws.meta, pred, host_log2, ws.max_log2);
  int rc = after_launch(ctx, "join_init_kernel");
  if (rc) return rc;
  const void* kb = reinterpret_cast<const void*>(&join_build_kernel<true>);
  join_build_kernel<true><<<grid_for(ctx, kb, kBuildBlock, 0, (nb + kBuildRowsPerThread - 1) / kBuildRowsPerThread),
                      kBuildBlock, 0, ctx->stream>>>(b, prm->date_lt, (uint32_t)prm->segment_eq, ws.slots, ws.bloom,
                                                     ws.meta, limit);
  if ((rc = after_launch(ctx, "join_build_kernel"))) return rc;
  for (int64_t c = 0; c < in.chunks; ++c) {
    const int64_t lo = c * kStreamChunkRows, n = std::max<int64_t>(0, std::min(np - lo, kStreamChunkRows));
    BO_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ev[3 + c], 0));
    const bo_join_probe_cols pc = {s.fk + lo, nullptr, nullptr, n};
    EmitOut eo;
    eo.rows = gs.rows_d + lo;
    eo.mult = gs.mult + lo;
    eo.counter = gs.counter + c;
    eo.count_host = gs.count_d + c;
    eo.capacity = (uint32_t)std::max<int64_t>(n, 0);
    if ((rc = launch_probe(ctx, pc, ws, s.part + c, mode, limit, false, eo))) return rc;
    BO_CUDA(ctx, cudaEventRecord(gs.probed[c], ctx->stream));
  }
  // Everything the task needs, by value: the set's buffers stay untouched
  // until the task has recorded the set's "done" event (the next query on the
  // set waits for the task's ticket first).
  const int64_t chunks = in.chunks;
  const std::vector<cudaEvent_t> probed(gs.probed.begin(), gs.probed.begin() + chunks);
  const uint32_t* rows_h = gs.rows_h;
  const volatile uint32_t* count_h = gs.count_h;
  const uint32_t* mult = gs.mult;
  const int64_t* price_h = ph->price;
  const int64_t* disc_h = ph->discount;
  bo_join_result* part = s.part;
  bo_join_result* combined = s.combined;
  const cudaEvent_t done_ev = ev[set];
  uint32_t* d_err = ctx->d_err;
  std::atomic<int64_t>* launches = &ctx->launches;
  const int max_grid = 2 * std::max(ctx->num_sms, 1);
  gs.ticket = g->queue.post([=](std::string& msg) -> int {
    GatherState& G = *g;
    auto fail = [&](cudaError_t e, const char* what) {
      msg = std::string(what) + ": " + cudaGetErrorString(e);
      return e == cudaErrorMemoryAllocation ? BO_ERR_OOM : BO_ERR_CUDA;
    };
    auto body = [&]() -> int {
      cudaError_t e;
      for (int64_t c = 0; c < chunks; ++c) {
        if ((e = cudaEventSynchronize(probed[c])) != cudaSuccess) return fail(e, "waiting for a probe chunk");
        const uint32_t n = count_h[c];
        if (n == 0) continue;
        if (n > (uint32_t)kStreamChunkRows) {
          msg = "match list longer than its chunk";
          return BO_ERR_DATA;
        }
        const int slot = G.next_rec;
        G.next_rec = (slot + 1) % kGatherRing;
        if (G.rec_busy[slot] && (e = cudaEventSynchronize(G.rec_ev[slot])) != cudaSuccess)
          return fail(e, "waiting for a staging buffer");
        const int64_t lo = c * kStreamChunkRows;
        const uint32_t* rows = rows_h + lo;
        const int64_t* pr = price_h + lo;
        const int64_t* dc = disc_h + lo;
        uint2* out = G.rec_h[slot];
        G.pool.parallel_for((int64_t)n, [&](int64_t b0, int64_t e0) { gather_rows(rows, pr, dc, out, b0, e0); });
        uint2* rec = G.rec_d + (size_t)slot * kStreamChunkRows;
        if ((e = cudaMemcpyAsync(rec, out, sizeof(uint2) * n, cudaMemcpyHostToDevice, G.stream)) != cudaSuccess)
          return fail(e, "copying gathered records");
        if ((e = cudaEventRecord(G.rec_ev[slot], G.stream)) != cudaSuccess) return fail(e, "recording a copy");
        G.rec_busy[slot] = true;
        const int grid = (int)std::min<int64_t>(max_grid, ((int64_t)n + 4 * kGatherBlock - 1) / (4 * kGatherBlock));
        join_gather_sum_kernel<<<grid, kGatherBlock, 0, G.stream>>>(rec, mult + lo, (int64_t)n, G.acc, part + c,
                                                                     d_err);
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "join_gather_sum_kernel");
        launches->fetch_add(1, std::memory_order_relaxed);
      }
      join_combine_kernel<<<1, 32, 0, G.stream>>>(part, chunks, combined);
      if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "join_combine_kernel");
      launches->fetch_add(1, std::memory_order_relaxed);
      if ((e = cudaMemcpyAsync(dst, combined, sizeof(bo_join_result), cudaMemcpyDeviceToHost, G.stream)) !=
          cudaSuccess)
        return fail(e, "copying the result");
      return 0;
    };
    const int rc2 = body();
    // The set's buffers are free once the gather stream gets here, also after a failure.
    const cudaError_t e = cudaEventRecord(done_ev, G.stream);
    if (!rc2 && e != cudaSuccess) return fail(e, "recording the set's done event");
    return rc2;
  });
  return BO_OK;
}

}  // namespace

int drain_host_work(bo_ctx* ctx) {
  GatherState* g = ctx ? ctx->gather : nullptr;
  if (!g) return BO_OK;
  std::string msg;
  const int rc = g->queue.drain(&msg);
  const cudaError_t e = g->stream ? cudaStreamSynchronize(g->stream) : cudaSuccess;
  if (rc) return set_error(ctx, rc, "join_stream gather: %s", msg.c_str());
  if (e != cudaSuccess) return cuda_fail(ctx, e, "gather stream");
  return BO_OK;
}

void destroy_host_work(bo_ctx* ctx) {
  GatherState* g = ctx ? ctx->gather : nullptr;
  if (!g) return;
  drain_host_work(ctx);
  free_gather(g);
  delete g;  // joins the queue's thread, then the pool's
  ctx->gather = nullptr;
}

}  // namespace bo

using namespace bo;

extern "C" {

int bo_join_count_device(bo_ctx* ctx, const bo_join_build_cols* b, const bo_join_params* prm, int64_t* count_device) {
  BO_CHECK_CTX(ctx);
  if (!b || !prm || !count_device) return set_error(ctx, BO_ERR_INVALID, "join_count: null argument");
  bo_join_probe_cols none = {};
  int rc = check_join(ctx, b, &none, prm);
  if (rc) return rc;
  BO_CUDA(ctx, cudaMemsetAsync(count_device, 0, sizeof(int64_t), ctx->stream));
  const void* kc = reinterpret_cast<const void*>(&join_count_kernel);
  const int gc = grid_for(ctx, kc, kBuildBlock, 0, (b->n_rows + 3) / 4);
  join_count_kernel<<<gc, kBuildBlock, 0, ctx->stream>>>(*b, prm->date_lt, (uint32_t)prm->segment_eq,
                                                          reinterpret_cast<unsigned long long*>(count_device));
  return after_launch(ctx, "join_count_kernel");
}

int bo_join_plain(bo_ctx* ctx, const bo_join_build_cols* b, const bo_join_probe_cols* p, const bo_join_params* prm,
                  bo_join_result* out_host) {
  BO_CHECK_CTX(ctx);
  int rc = check_join(ctx, b, p, prm);
  if (rc) return rc;
  if (!out_host) return set_error(ctx, BO_ERR_INVALID, "join: null output");
  return join_plain_impl(ctx, *b, *p, *prm, out_host, 0);
}

int bo_join_presized_device(bo_ctx* ctx, const bo_join_build_cols* b, const bo_join_probe_cols* p,
                            const bo_join_params* prm, const float* pred_device, bo_join_result* out_device) {
  BO_CHECK_CTX(ctx);
  int rc = check_join(ctx, b, p, prm);
  if (rc) return rc;
  if (!pred_device || !out_device) return set_error(ctx, BO_ERR_INVALID, "join: null prediction or output");
  JoinWs ws;
  if ((rc = join_workspace(ctx, b->n_rows, &ws))) return rc;
  return join_run(ctx, *b, *p, *prm, ws, pred_device, 0, out_device, 1);
}

int bo_join_learned_device(bo_ctx* ctx, const bo_mlp* m, const float* features_host, const bo_join_build_cols* b,
                           const bo_join_probe_cols* p, const bo_join_params* prm, bo_join_result* out_device,
                           float* pred_device) {
  BO_CHECK_CTX(ctx);
  int rc = check_join(ctx, b, p, prm);
  if (rc) return rc;
  const float* params = nullptr;
  int F = 0, O = 0;
  if (!features_host || !out_device || mlp_view(m, &params, &F, &O) != BO_OK || F < 1 || F > kMaxF || O < 1 ||
      O > kMaxO)
    return set_error(ctx, BO_ERR_INVALID, "join_learned: null argument or bad model");
  FeatureVec fv;
  for (int i = 0; i < kMaxF; ++i) fv.f[i] = i < F ? features_host[i] : 0.0f;
  JoinWs ws;
  if ((rc = join_workspace(ctx, b->n_rows, &ws))) return rc;
  join_learned_init_kernel<<<ctx->num_sms * 2, kPredThreads, 0, ctx->stream>>>(params, fv, F, O, ws.slots, ws.bloom,
                                                                             ws.meta, ws.max_log2, pred_device);
  if ((rc = after_launch(ctx, "join_learned_init_kernel"))) return rc;
  const void* kb = reinterpret_cast<const void*>(&join_build_kernel<false>);
  const int gb = grid_for(ctx, kb, kBuildBlock, 0, (b->n_rows + kBuildRowsPerThread - 1) / kBuildRowsPerThread);
  BO_CUDA(ctx, launch_dependent(&join_build_kernel<false>, gb, kBuildBlock, 0, ctx->stream, *b, prm->date_lt,
                                (uint32_t)prm->segment_eq, ws.slots, ws.bloom, ws.meta, (uint64_t)kPresizedProbeLimit));
  if ((rc = after_launch(ctx, "join_build_kernel"))) return rc;
  return launch_probe(ctx, *p, ws, out_device, 1, kPresizedProbeLimit, true);
}

int bo_join_learned(bo_ctx* ctx, const bo_mlp* m, const float* features_host, const bo_join_build_cols* b,
                    const bo_join_probe_cols* p, const bo_join_params* prm, bo_join_result* out_host) {
  BO_CHECK_CTX(ctx);
  if (!out_host) return set_error(ctx, BO_ERR_INVALID, "join: null output");
  void* dout = nullptr;
  int rc = region(ctx, "join_out", sizeof(bo_join_result), &dout);
  if (rc) return rc;
  bo_join_result* d = static_cast<bo_join_result*>(dout);
  if ((rc = bo_join_learned_device(ctx, m, features_host, b, p, prm, d, nullptr))) return rc;
  if ((rc = finish_join(ctx, out_host, d))) return rc;
  if (out_host->overflowed) {  // the prediction was too low: the exact form
    if ((rc = join_plain_impl(ctx, *b, *p, *prm, out_host, 1))) return rc;
    out_host->mode = 1;
  }
  return BO_OK;
}

int bo_join_presized(bo_ctx* ctx, const bo_join_build_cols* b, const bo_join_probe_cols* p, const bo_join_params* prm,
                     const float* pred_device, bo_join_result* out_host) {
  BO_CHECK_CTX(ctx);
  if (!out_host) return set_error(ctx, BO_ERR_INVALID, "join: null output");
  void* dout = nullptr;
  int rc = region(ctx, "join_out", sizeof(bo_join_result), &dout);
  if (rc) return rc;
  bo_join_result* d = static_cast<bo_join_result*>(dout);
  if ((rc = bo_join_presized_device(ctx, b, p, prm, pred_device, d))) return rc;
  if ((rc = finish_join(ctx, out_host, d))) return rc;
  if (out_host->overflowed) {
    // The prediction was too low: rerun exactly (the answer never depends on it).
    const int32_t cap = out_host->capacity_log2;
    if ((rc = join_plain_impl(ctx, *b, *p, *prm, out_host, 1))) return rc;
    out_host->mode = 1;
    (void)cap;
  }
  return BO_OK;
}

int bo_join_probe_device(bo_ctx* ctx, const bo_join_probe_cols* p, bo_join_result* out_device) {
  BO_CHECK_CTX(ctx);
  if (!p || !out_device) return set_error(ctx, BO_ERR_INVALID, "join_probe: null argument");
  if (p->n_rows < 0) return set_error(ctx, BO_ERR_INVALID, "join_probe: negative row count");
  if (p->n_rows > 0 && (!p->fk || !p->price || !p->discount || !aligned32(p->fk) || !aligned32(p->price) ||
                        !aligned32(p->discount)))
    return set_error(ctx, BO_ERR_INVALID, "join_probe: probe column null or not 32-byte aligned");
  auto it = ctx->regions.find("join_slots");
  if (it == ctx->regions.end())
    return set_error(ctx, BO_ERR_INVALID, "join_probe: no join table has been built on this context");
  JoinWs ws;
  int rc = join_workspace(ctx, 0, &ws);
  if (rc) return rc;
  return launch_probe(ctx, *p, ws, out_device, 1, ~0ull);  // the table's build bound is not known here
}

int bo_join_host(bo_ctx* ctx, const bo_join_build_cols* bh, const bo_join_probe_cols* ph, const bo_join_params* prm,
                 int32_t mode, float predicted_rows, bo_join_result* out_host) {
  BO_CHECK_CTX(ctx);
  if (!bh || !ph || !prm || !out_host) return set_error(ctx, BO_ERR_INVALID, "join: null argument");
  if (bh->n_rows < 0 || ph->n_rows < 0) return set_error(ctx, BO_ERR_INVALID, "join: negative row count");
  const size_t nb = (size_t)bh->n_rows, np = (size_t)ph->n_rows;
  const size_t sizes[6] = {4 * nb, 4 * nb, nb, 4 * np, 8 * np, 8 * np};
  const void* src[6] = {bh->key, bh->date, bh->segment, ph->fk, ph->price, ph->discount};
  size_t off[6], total = 0;
  for (int i = 0; i < 6; ++i) {
    off[i] = total;
    total += (sizes[i] + 255) & ~size_t(255);
  }
  void* base = nullptr;
  int rc = region(ctx, "join_in", total ? total : 256, &base);
  if (rc) return rc;
  char* d = static_cast<char*>(base);
  for (int i = 0; i < 6; ++i)
    if (sizes[i]) BO_CUDA(ctx, cudaMemcpyAsync(d + off[i], src[i], sizes[i], cudaMemcpyHostToDevice, ctx->stream));
  bo_join_build_cols b = {reinterpret_cast<const int32_t*>(d + off[0]), reinterpret_cast<const int32_t*>(d + off[1]),
                          reinterpret_cast<const uint8_t*>(d + off[2]), bh->n_rows};
  bo_join_probe_cols p = {reinterpret_cast<const int32_t*>(d + off[3]), reinterpret_cast<const int64_t*>(d + off[4]),
                          reinterpret_cast<const int64_t*>(d + off[5]), ph->n_rows};
  if (mode == 0) return bo_join_plain(ctx, &b, &p, prm, out_host);
  JoinWs ws;
  if ((rc = join_workspace(ctx, b.n_rows, &ws))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(ws.pred, &predicted_rows, sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  return bo_join_presized(ctx, &b, &p, prm, ws.pred, out_host);
}

// Streamed join over pinned host columns (see include/bespoke_gpu.h).
int bo_join_stream_host(bo_ctx* ctx, const bo_join_build_cols* bh, const bo_join_probe_cols* ph,
                        const bo_join_params* prm, const float* pred_device, bo_join_result* out_host) {
  BO_CHECK_CTX(ctx);
  if (!out_host) return set_error(ctx, BO_ERR_INVALID, "join_stream: null output");
  StreamIn in;
  int rc = stream_check(ctx, bh, ph, prm, &in);
  if (rc) return rc;
  GatherState* g = nullptr;
  if ((rc = gather_state(ctx, &g))) return rc;
  JoinWs ws;
  StreamSet s;
  const int set = ctx->stream_set ^= 1;
  if (g) {  // the set's previous query must have handed its buffers back first
    g->queue.wait_for(g->set[set].ticket);
    if ((rc = gather_reserve(ctx, g, ph->n_rows, in.chunks))) return rc;
  }
  if ((rc = join_workspace(ctx, bh->n_rows, &ws)) || (rc = stream_set(ctx, bh->n_rows, ph->n_rows, in.chunks, set, &s)) ||
      (rc = stream_events(ctx, in.chunks)) || (rc = stream_copies(ctx, bh, ph, in, s, set)))
    return rc;
  int32_t cl = 0;
  if (!pred_device) {  // exact-count form: one host round trip, as bo_join_plain
    BO_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->events[2], 0));
    const bo_join_build_cols b = {in.key, s.date, s.seg, bh->n_rows};
    BO_CUDA(ctx, cudaMemsetAsync(&ws.meta->count, 0, sizeof(unsigned long long), ctx->stream));
    const void* kc = reinterpret_cast<const void*>(&join_count_kernel);
    join_count_kernel<<<grid_for(ctx, kc, kBuildBlock, 0, (bh->n_rows + 3) / 4), kBuildBlock, 0, ctx->stream>>>(
        b, prm->date_lt, (uint32_t)prm->segment_eq, &ws.meta->count);
    if ((rc = after_launch(ctx, "join_count_kernel"))) return rc;
    unsigned long long count = 0;
    BO_CUDA(ctx, cudaMemcpyAsync(&count, &ws.meta->count, sizeof(count), cudaMemcpyDeviceToHost, ctx->stream));
    BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    cl = std::min(ws.max_log2, std::max(kMinCapLog2, ceil_log2(std::max<uint64_t>(count, 1) * kPlainSlotsPerRow)));
  }
  if (g) {
    if ((rc = stream_compute_gather(ctx, g, bh, ph, prm, pred_device, cl, ws, in, s, set, g->set[set].res_h)))
      return rc;
  } else {
    if ((rc = stream_compute(ctx, bh, ph, prm, pred_device, cl, ws, in, s, set))) return rc;
    BO_CUDA(ctx, cudaMemcpyAsync(out_host, s.combined, sizeof(bo_join_result), cudaMemcpyDeviceToHost, ctx->stream));
  }
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // drains the gather, synchronises the stream
  if ((rc = device_error_status(ctx, bits, "join_stream"))) return rc;
  if (g) *out_host = *g->set[set].res_h;
  out_host->mode = pred_device ? 1 : 0;
  if (out_host->overflowed && pred_device) {  // the prediction was too low: rerun with the exact count
    if ((rc = bo_join_stream_host(ctx, bh, ph, prm, nullptr, out_host))) return rc;
    out_host->reruns = 1;
    out_host->mode = 1;
    return BO_OK;
  }
  if (out_host->overflowed) return set_error(ctx, BO_ERR_OVERFLOW, "join_stream: exact-size table overflowed");
  return BO_OK;
}

int bo_join_stream_host_async(bo_ctx* ctx, const bo_join_build_cols* bh, const bo_join_probe_cols* ph,
                              const bo_join_params* prm, const float* pred_device, bo_join_result* out_pinned) {
  BO_CHECK_CTX(ctx);
  if (!pred_device || !out_pinned) return set_error(ctx, BO_ERR_INVALID, "join_stream_async: null prediction/output");
  if (!mapped_device_pointer(out_pinned))
    return set_error(ctx, BO_ERR_INVALID, "join_stream_async: the result must be pinned host memory");
  StreamIn in;
  int rc = stream_check(ctx, bh, ph, prm, &in);
  if (rc) return rc;
  GatherState* g = nullptr;
  if ((rc = gather_state(ctx, &g))) return rc;
  JoinWs ws;
  StreamSet s;
  const int set = ctx->stream_set ^= 1;
  if (g) {  // the set's previous query must have handed its buffers back first
    g->queue.wait_for(g->set[set].ticket);
    if ((rc = gather_reserve(ctx, g, ph->n_rows, in.chunks))) return rc;
  }
  if ((rc = join_workspace(ctx, bh->n_rows, &ws)) || (rc = stream_set(ctx, bh->n_rows, ph->n_rows, in.chunks, set, &s)) ||
      (rc = stream_events(ctx, in.chunks)) || (rc = stream_copies(ctx, bh, ph, in, s, set)))
    return rc;
  if (g) return stream_compute_gather(ctx, g, bh, ph, prm, pred_device, 0, ws, in, s, set, out_pinned);
  if ((rc = stream_compute(ctx, bh, ph, prm, pred_device, 0, ws, in, s, set))) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(out_pinned, s.combined, sizeof(bo_join_result), cudaMemcpyDeviceToHost, ctx->stream));
  return BO_OK;
}

int bo_set_host_threads(bo_ctx* ctx, int32_t threads) {
  BO_CHECK_CTX(ctx);
  if (threads > 256) return set_error(ctx, BO_ERR_INVALID, "set_host_threads: %d threads", threads);
  const int t = threads < 0 ? -1 : threads;
  if (t == ctx->gather_threads) return BO_OK;
  if (int rc = drain_host_work(ctx)) return rc;
  destroy_host_work(ctx);  // recreated with the new count by the next streamed join
  ctx->gather_threads = t;
  return BO_OK;
}

int bo_host_threads(const bo_ctx* ctx) {
  if (!ctx) return 0;
  return ctx->gather_threads < 0 ? auto_gather_threads() : ctx->gather_threads;
}

}  // extern "C"
