// Batched heterogeneous pipelines: one persistent kernel over a device work
// queue, captured in a CUDA graph.
//
// The reference answers one query per call (bespoke_tpch/query_impl.cpp:159-388
// dispatches a single run_qN per request); batching many pipelines into one
// launch has no reference counterpart.  Every stage below computes with the same
// per-row code as the standalone kernels (rows.cuh), so each instance's answer is
// the one its solo run gives.
//
// Work items.  An instance's pipeline is a short chain of stages; each stage is
// cut into tiles (row ranges, slot ranges or bitmap-word ranges) and every tile
// is one work item (instance, stage, level, tile).  The host orders the items
// level-major (all first stages, then all second stages, ...; larger instances
// first inside a level) and the kernel's blocks pop them from a global counter
// in that order.  A tile at level l of an instance waits -- bounded by the
// global timer -- until every level l-1 tile of that instance has signalled
// completion.  Items are only popped by running blocks and every item an item
// waits for sits earlier in the queue, so some block always makes progress.
//
// Stages (level):
//   scan-agg  0 Q1 scan tile: per-thread shared-memory group columns, flushed
//               into the instance's 128-bit totals; the last tile (ticket)
//               writes the records;
//   join      0 init (clear slots; tile 0 the Bloom filter)
//             1 build tile (filter, CAS insert, Bloom bits)
//             2 probe tile (Bloom filter TMA-staged in shared memory once per
//               block and instance, warp queues, late materialisation); the
//               last tile writes the result;
//   group-by  0 init (slots, minima, A mask; tile 0 the Bloom filter)
//             1 C filter tile (exact bitmap + Bloom bits) and A mask tile
//             2 B scan tile (Bloom, exact bitmap, A mask, shared pre-aggregation
//               table, global CAS table)
//             3 select tile: the k smallest packed (count desc, id asc) keys of a
//               slot range by a block radix select; the last tile merges the
//               tiles' candidates and writes the ordered top-k.
// Tables are sized on the host from each instance's prediction; an instance
// whose table overflowed is rerun alone in the exact form when results are read.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "context.cuh"
#include "rows.cuh"

namespace bo {
namespace {

constexpr int kBB = 256;  // threads per worker block
constexpr int kBW = kBB / 32;
constexpr int kLevels = 4;
constexpr uint32_t kScratchBytes = 32 * 1024;
constexpr uint32_t kSmemBytes = kBloomBytes + kScratchBytes;  // region A (Bloom / Q1 columns) + region B
static_assert(kBB == kScanBlock, "the scan-agg columns are laid out for kScanBlock threads");
static_assert(BO_BATCH_MAX_CATS == 64, "category set size");

enum Stage : int {
  kSQ1 = 0,
  kSJInit,
  kSJBuild,
  kSJProbe,
  kSGInit,
  kSGCFilter,
  kSGAMask,
  kSGScan,
  kSGSelect,
  kNumStages
};
constexpr int kStageLevel[kNumStages] = {0, 0, 1, 2, 0, 1, 1, 2, 3};

// Rows of one scan-agg flush period: <= 63 four-row chunks per thread plus one
// tail row keeps every per-thread packed field inside its bits.
constexpr int64_t kQ1SubRows = (int64_t)((kMaxRowsPerThread - 1) / 4) * 4 * kBB;
// Tile sizing: a stage of n units is cut into about kTargetTiles tiles (two per
// worker block of a 148-SM B200 at two blocks per SM), so that even a lone large
// instance spreads every stage over the whole GPU, but never into tiles below
// the stage's minimum (per-item overhead) nor above the autotuned maximum.
constexpr int64_t kTargetTiles = 2 * 148 * 2;
constexpr int64_t kPoolMaxParticipants = 2 * 148;     // one per worker block
constexpr int64_t kPoolWarps = kPoolMaxParticipants * 8;
constexpr int64_t kPoolChunksPerWarp = 4;
constexpr int64_t kPoolChunksPerBlock = 16;
constexpr int kSelChunk = 1024;   // slots (or candidates) added per select round
constexpr int kSelBuf = 2048;     // select buffer entries
constexpr int kQ1ColBytes = BO_Q1_MAX_GROUPS * kWideWords * kBB * 8;
static_assert(kQ1ColBytes + kBW * BO_Q1_MAX_GROUPS * kQ1Sums * 8 <= (int)kSmemBytes, "scan-agg columns fit");
constexpr int kProbeResolveB = 4;  // join candidates per lane per resolve round
constexpr int kGbQueueB = 384;
constexpr int kGbFlushAtB = 128;
constexpr int kGbResolveB = 4;
constexpr int kGbLocalB = 256;
constexpr int kGbLocalProbesB = 2;

struct InstDesc {
  int32_t kind;
  int32_t cap_log2;          // table capacity (the upper bound when pred_dev is set)
  const float* pred_dev;     // optional device prediction read at launch time
  float factor;              // slots per predicted row
  uint32_t level_items[kLevels];
  int64_t unit[kNumStages];       // rows / slots / words per tile (fixed stages) or chunk (pooled stages)
  uint32_t n_chunks[kNumStages];  // chunks of a pooled stage (= tiles of a fixed stage)
  uint32_t n_tiles[kNumStages];   // work items: tiles of a fixed stage, participants of a pooled one
  // scan-agg
  bo_fact_cols fact;
  int32_t cutoff;
  uint32_t n_fa, n_fb;
  // join
  bo_join_build_cols build;
  bo_join_probe_cols probe;
  int32_t date_lt;
  uint32_t seg;
  // group-by
  bo_gb_a_cols a;
  bo_gb_b_cols b;
  bo_gb_c_cols c;
  uint16_t cats[BO_BATCH_MAX_CATS];
  int32_t n_cats, year_lo, year_hi, k, a_id_max, wa;
  unsigned long long cmax;
  int64_t mask_words, c_words;
  // tables (device)
  unsigned long long* slots;
  int32_t* mins;
  uint32_t* bloom;
  uint32_t* cbits;
  uint32_t* amask;
  unsigned long long* cand_keys;
  uint32_t* cand_vals;
};

// Per-instance state, zeroed at the start of every launch.
struct InstState {
  uint32_t done[kLevels];  // completed items per level
  uint32_t ticket;         // finishing ticket of the last stage
  uint32_t overflow;
  uint32_t cursor[kNumStages];  // next chunk of each pooled stage
  uint32_t pad[1];
  // join: 0 build rows, 1 distinct keys; group-by: 0 joined, 1 distinct, 2 C passing, 3 groups
  unsigned long long cnt[4];
  unsigned long long n_cand;
  unsigned long long pad2[3];
  unsigned long long acc[BO_Q1_MAX_GROUPS * kQ1Sums * 2];  // scan-agg 128-bit totals; join uses [0, 6)
};
static_assert(sizeof(InstState) % 64 == 0, "state alignment");

// ------------------------------------------------------------- helpers ----
__device__ __forceinline__ uint64_t warp_or_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block sum of three counters and an OR flag; thread 0 gets the totals.
__device__ __forceinline__ void block_counts(uint32_t a, uint32_t b, uint32_t c, uint32_t f, uint32_t (*red)[kBW],
                                             uint32_t out[4]) {
  const uint32_t wa = warp_sum_u32(a), wb = warp_sum_u32(b), wc = warp_sum_u32(c);
  const uint32_t wf = __any_sync(0xffffffffu, f != 0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = wa;
    red[1][warp] = wb;
    red[2][warp] = wc;
    red[3][warp] = wf;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    out[0] = out[1] = out[2] = out[3] = 0;
    for (int w = 0; w < kBW; ++w) {
      out[0] += red[0][w];
      out[1] += red[1][w];
      out[2] += red[2][w];
      out[3] |= red[3][w];
    }
  }
  __syncthreads();
}

// Ticket of a stage's finishing tile: true in every thread of the block that
// completed the stage's last tile (all other tiles' writes are then visible).
__device__ __forceinline__ bool last_tile(uint32_t* ticket, uint32_t n_tiles, uint32_t* flag) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) *flag = (atomicAdd(ticket, 1u) == n_tiles - 1u) ? 1u : 0u;
  __syncthreads();
  const bool last = *flag != 0u;
  if (last) __threadfence();
  return last;
}

// ------------------------------------------------------ block top-k select --
// Keeps the k smallest of a stream of unique 64-bit keys (with a 32-bit value)
// in shared memory.  Keys enter a buffer only if below the current k-th
// smallest; when the buffer passes kSelChunk entries a block radix select (8-bit
// digits from the highest bit in which the keys differ) cuts it back to k.
struct SelCtl {
  unsigned long long bound;  // keys >= bound cannot be among the k smallest
  unsigned long long diff;
  unsigned long long tmax;
  uint32_t n;
  uint32_t pos;
  uint32_t d, before, cnt;
};

struct SelBuf {
  unsigned long long* keys;  // kSelBuf
  uint32_t* vals;            // kSelBuf
  uint32_t* hist;            // 256
  SelCtl* ctl;
};

__device__ __forceinline__ unsigned long long hi_bits(unsigned long long key, int s) {
  return s >= 64 ? 0ull : (key >> s);
}

__device__ __forceinline__ void sel_reset(SelBuf& sb) {
  if (threadIdx.x == 0) {
    sb.ctl->bound = ~0ull;
    sb.ctl->n = 0;
  }
  __syncthreads();
}

// Warp-aggregated append of the lanes whose `ok` is set (call from all lanes).
__device__ __forceinline__ void sel_add(SelBuf& sb, bool ok, unsigned long long key, uint32_t val,
                                        unsigned long long bound) {
  ok = ok && key < bound;
  const uint32_t m = __ballot_sync(0xffffffffu, ok);
  if (m == 0u) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&sb.ctl->n, (uint32_t)__popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (ok) {
    const uint32_t p = base + __popc(m & ((1u << lane) - 1u));
    sb.keys[p] = key;
    sb.vals[p] = val;
  }
}

// Cuts the buffer to its k smallest keys (unordered) and sets the bound.
// Block-uniform; n = sb.ctl->n must be read after a barrier.
__device__ void sel_reduce(SelBuf& sb, int k) {
  __syncthreads();
  const uint32_t n = sb.ctl->n;
  if (n <= (uint32_t)k) return;
  if (k == 0) {
    __syncthreads();
    if (threadIdx.x == 0) {
      sb.ctl->n = 0;
      sb.ctl->bound = 0ull;
    }
    __syncthreads();
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    sb.ctl->diff = 0ull;
    sb.ctl->tmax = 0ull;
    sb.ctl->pos = 0u;
  }
  __syncthreads();
  const unsigned long long k0 = sb.keys[0];
  unsigned long long dl = 0;
  for (uint32_t i = threadIdx.x; i < n; i += kBB) dl |= sb.keys[i] ^ k0;
  dl = warp_or_u64(dl);
  if (lane == 0 && dl) atomicOr(&sb.ctl->diff, dl);
  __syncthreads();
  const unsigned long long diff = sb.ctl->diff;  // != 0: n >= 2 distinct keys
  int shift = ((63 - __clzll((long long)diff)) / 8) * 8;
  unsigned long long prefix = hi_bits(k0, shift + 8);
  uint32_t need = (uint32_t)k;
  for (;;) {
    sb.hist[threadIdx.x] = 0u;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += kBB) {
      const unsigned long long key = sb.keys[i];
      if (hi_bits(key, shift + 8) == prefix) atomicAdd(&sb.hist[(key >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (warp == 0) {
      uint32_t h[8], s = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        h[j] = sb.hist[8 * lane + j];
        s += h[j];
      }
      uint32_t incl = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      const uint32_t excl = incl - s;
      if (excl < need && need <= incl) {
        uint32_t c = excl;
#pragma unroll 1
        for (int j = 0; j < 8; ++j) {
          if (c + h[j] >= need) {
            sb.ctl->d = (uint32_t)(8 * lane + j);
            sb.ctl->before = c;
            sb.ctl->cnt = h[j];
            break;
          }
          c += h[j];
        }
      }
    }
    __syncthreads();
    const uint32_t d = sb.ctl->d, before = sb.ctl->before, cnt = sb.ctl->cnt;
    need -= before;
    prefix = (prefix << 8) | d;
    if (cnt == need || shift == 0) break;  // (keys are unique: cnt == need at shift 0)
    shift -= 8;
    __syncthreads();
  }
  // Gather the selected keys (hi_bits <= prefix) to the front.
  unsigned long long rk[kSelBuf / kBB];
  uint32_t rv[kSelBuf / kBB];
#pragma unroll
  for (int j = 0; j < kSelBuf / kBB; ++j) {
    const uint32_t i = threadIdx.x + j * kBB;
    rk[j] = i < n ? sb.keys[i] : ~0ull;
    rv[j] = i < n ? sb.vals[i] : 0u;
  }
  __syncthreads();
  unsigned long long tmax = 0ull;
#pragma unroll
  for (int j = 0; j < kSelBuf / kBB; ++j) {
    const uint32_t i = threadIdx.x + j * kBB;
    if (i < n && hi_bits(rk[j], shift) <= prefix) {
      const uint32_t p = atomicAdd(&sb.ctl->pos, 1u);
      if (p < (uint32_t)k) {
        sb.keys[p] = rk[j];
        sb.vals[p] = rv[j];
      }
      tmax = rk[j] > tmax ? rk[j] : tmax;
    }
  }
  if (tmax) atomicMax(&sb.ctl->tmax, tmax);
  __syncthreads();
  if (threadIdx.x == 0) {
    sb.ctl->n = min(sb.ctl->pos, (uint32_t)k);
    sb.ctl->bound = sb.ctl->tmax;
  }
  __syncthreads();
}

// --------------------------------------------------------------- stages ---
struct Smem {
  unsigned char* a;  // region A: Bloom filter or scan-agg columns
  unsigned char* b;  // region B: stage scratch
};

// Scan-agg tile (wide layout), flushed every kQ1SubRows rows.
__device__ void stage_q1(const InstDesc& d, InstState* st, uint32_t tile, const Smem& sm, bo_batch_result* res,
                         uint32_t* flag, uint32_t* err) {
  unsigned long long* col = reinterpret_cast<unsigned long long*>(sm.a) + threadIdx.x;
  int64_t* warp_part = reinterpret_cast<int64_t*>(sm.a + kQ1ColBytes);
  const int ng = (int)(d.n_fa * d.n_fb);
  const bo_fact_cols& c = d.fact;
  const int64_t n = c.n_rows;
  const int64_t lo = (int64_t)tile * d.unit[kSQ1];
  const int64_t hi = min(n, lo + d.unit[kSQ1]);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t bad = 0;
  for (int64_t r = lo; r < hi; r += kQ1SubRows) {
    const int64_t sh = min(hi, r + kQ1SubRows);
#pragma unroll 1
    for (int i = 0; i < ng * kWideWords; ++i) col[i * kBB] = 0ull;
    for (int64_t ch = (r >> 2) + threadIdx.x; ch < (sh >> 2); ch += kBB) {
      const int64_t rr = ch << 2;
      const int4 sd = ld_stream_v4(c.ship_date + rr);
      const long4v q = ld_stream_v4x64(c.quantity + rr), p = ld_stream_v4x64(c.ext_price + rr);
      const long4v dd = ld_stream_v4x64(c.discount + rr), t = ld_stream_v4x64(c.tax + rr);
      const uint32_t fa = ld_stream_u32(c.flag_a + rr), fb = ld_stream_u32(c.flag_b + rr);
      const int32_t ship[4] = {sd.x, sd.y, sd.z, sd.w};
#pragma unroll
      for (int k = 0; k < 4; ++k)
        wide_row(col, ship[k], d.cutoff, q.v[k], p.v[k], dd.v[k], t.v[k], (fa >> (8 * k)) & 0xffu,
                 (fb >> (8 * k)) & 0xffu, d.n_fa, d.n_fb, bad);
    }
    const int64_t tail = ((sh >> 2) << 2) + threadIdx.x;  // only the table's last rows
    if (tail < sh && tail >= r) {
      wide_row(col, c.ship_date[tail], d.cutoff, c.quantity[tail], c.ext_price[tail], c.discount[tail], c.tax[tail],
               c.flag_a[tail], c.flag_b[tail], d.n_fa, d.n_fb, bad);
    }
    // Block reduction into the instance's 128-bit totals.
#pragma unroll 1
    for (int g = 0; g < ng; ++g) {
      int64_t v[kQ1Sums];
      wide_canon(col, g, v);
#pragma unroll
      for (int s = 0; s < kQ1Sums; ++s) {
        const int64_t w = warp_sum_i64(v[s]);
        if (lane == 0) warp_part[warp * (BO_Q1_MAX_GROUPS * kQ1Sums) + g * kQ1Sums + s] = w;
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ng * kQ1Sums; i += kBB) {
      __int128 tot = 0;
      for (int w = 0; w < kBW; ++w) tot += (__int128)warp_part[w * (BO_Q1_MAX_GROUPS * kQ1Sums) + i];
      if (tot != 0) atomic_add_i128(st->acc + 2 * i, tot);
    }
    __syncthreads();
  }
  if (bad) raise_error(err, bad);
  if (last_tile(&st->ticket, d.n_tiles[kSQ1], flag)) {
    uint32_t fbad = 0;
    if (threadIdx.x < ng) {
      __int128 t[kQ1Sums];
#pragma unroll
      for (int s = 0; s < kQ1Sums; ++s) t[s] = load_i128(st->acc + 2 * (threadIdx.x * kQ1Sums + s));
      res->q1[threadIdx.x] = q1_record(t, fbad);
    }
    if (threadIdx.x == 0) {
      res->kind = BO_BATCH_SCAN_AGG;
      res->overflowed = 0;
      res->reruns = 0;
    }
    if (fbad) raise_error(err, fbad);
  }
}

// Slot range [lo, hi) of tile t when `total` entries are split over n tiles.
__device__ __forceinline__ void split_range(int64_t total, uint32_t t, uint32_t n, int64_t& lo, int64_t& hi) {
  lo = (int64_t)((__int128)total * t / n);
  hi = (int64_t)((__int128)total * (t + 1) / n);
}

// Capacity of this launch: planned on the host, or derived on the device from
// a prediction in device memory by the solo presized forms' rule (smallest
// power of two >= factor * prediction, at least 2^10, at most the planned
// upper bound).  Every tile computes the same value from the same float.
__device__ __forceinline__ int32_t cap_log2_of(const InstDesc& d) {
  if (!d.pred_dev) return d.cap_log2;
  float p = __ldcg(d.pred_dev);
  if (!(p >= 0.0f)) p = 0.0f;
  const double want = (double)p * d.factor;
  int32_t cl = 10;
  while (cl < d.cap_log2 && (double)(1ull << cl) < want) ++cl;
  return cl;
}

// Streaming stages run as chunk pools: an instance's stage has a few
// participant items (blocks); each warp of a participant takes the stage's
// next chunk from a per-instance cursor until none are left, so work spreads
// evenly over warps and blocks whatever the stage's size, and the block-level
// totals are flushed once per participant rather than once per chunk.
__device__ __forceinline__ bool next_chunk(uint32_t* cursor, uint32_t n_chunks, uint32_t& c) {
  uint32_t v = 0;
  if ((threadIdx.x & 31) == 0) v = atomicAdd(cursor, 1u);
  c = __shfl_sync(0xffffffffu, v, 0);
  return c < n_chunks;
}

// Units [lo, hi) of chunk c, clipped to n.
__device__ __forceinline__ void chunk_range(uint32_t c, int64_t unit, int64_t n, int64_t& lo, int64_t& hi) {
  lo = (int64_t)c * unit;
  hi = min(n, lo + unit);
}

__device__ __forceinline__ unsigned __int128 warp_sum_u128(unsigned __int128 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long lo = __shfl_xor_sync(0xffffffffu, (unsigned long long)v, o);
    const unsigned long long hi = __shfl_xor_sync(0xffffffffu, (unsigned long long)(v >> 64), o);
    v += ((unsigned __int128)hi << 64) | lo;
  }
  return v;
}

__device__ void stage_join_init(const InstDesc& d, InstState* st, uint32_t part) {
  const int64_t cap = (int64_t)1 << cap_log2_of(d);
  if (part == 0) {
    uint4* b4 = reinterpret_cast<uint4*>(d.bloom);
    for (uint32_t i = threadIdx.x; i < kBloomWords / 4; i += kBB) b4[i] = make_uint4(0, 0, 0, 0);
  }
  ulonglong2* s2 = reinterpret_cast<ulonglong2*>(d.slots);
  const int lane = threadIdx.x & 31;
  uint32_t c;
  while (next_chunk(&st->cursor[kSJInit], d.n_chunks[kSJInit], c)) {
    int64_t lo, hi;
    chunk_range(c, d.unit[kSJInit], cap, lo, hi);  // even bounds: unit and cap are even
    for (int64_t i = lo / 2 + lane; i < hi / 2; i += 32) s2[i] = make_ulonglong2(kEmptySlot, kEmptySlot);
  }
}

__device__ void stage_join_build(const InstDesc& d, InstState* st, const Smem& sm, uint32_t (*red)[kBW]) {
  const bo_join_build_cols b = d.build;
  const int32_t date_lt = d.date_lt;
  const uint32_t seg = d.seg;
  unsigned long long* slots = d.slots;
  uint32_t* bloom = d.bloom;
  const uint64_t mask = (1ull << cap_log2_of(d)) - 1;
  const int lane = threadIdx.x & 31;
  uint32_t* bq = reinterpret_cast<uint32_t*>(sm.b) + (threadIdx.x >> 5) * 256;
  uint32_t qual = 0, newkeys = 0;
  bool full = false;
  uint32_t c;
  while (next_chunk(&st->cursor[kSJBuild], d.n_chunks[kSJBuild], c)) {
    int64_t lo, hi;
    chunk_range(c, d.unit[kSJBuild], b.n_rows, lo, hi);
    for (int64_t base = lo; base < hi; base += 512) {  // warp-uniform: 16 rows per lane
      const int64_t r0 = base + lane * 16;
      uint32_t q = 0;
      if (r0 + 16 <= hi) {
        const int4 sg = ld_stream_v4(b.segment + r0);
        const uint32_t sw[4] = {(uint32_t)sg.x, (uint32_t)sg.y, (uint32_t)sg.z, (uint32_t)sg.w};
        const int8v d0 = ld_stream_v8(b.date + r0), d1 = ld_stream_v8(b.date + r0 + 8);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int32_t dk = k < 8 ? d0.v[k] : d1.v[k - 8];
          q |= (uint32_t)build_qual(dk, (sw[k >> 2] >> (8 * (k & 3))) & 0xffu, date_lt, seg) << k;
        }
      } else {
        for (int k = 0; k < 16; ++k)
          if (r0 + k < hi && build_qual(b.date[r0 + k], b.segment[r0 + k], date_lt, seg)) q |= 1u << k;
      }
      qual += __popc(q);
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const uint32_t hm = (q >> (8 * half)) & 0xffu;
        uint32_t total;
        uint32_t pos = warp_exclusive_scan(__popc(hm), total);
        if (total == 0) continue;
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if ((hm >> k) & 1u) bq[pos++] = (uint32_t)(lane * 16 + 8 * half + k);
        __syncwarp();
        for (uint32_t i = lane; i < total; i += 32)
          join_insert(slots, bloom, mask, __ldg(b.key + base + bq[i]), newkeys, full, kPresizedProbeLimit);
        __syncwarp();
      }
    }
  }
  uint32_t tot[4];
  block_counts(qual, newkeys, 0, full, red, tot);
  if (threadIdx.x == 0) {
    if (tot[0]) atomicAdd(&st->cnt[0], (unsigned long long)tot[0]);
    if (tot[1]) {
      const unsigned long long before = atomicAdd(&st->cnt[1], (unsigned long long)tot[1]);
      if (before + tot[1] > (mask + 1) - ((mask + 1) >> 3)) atomicOr(&st->overflow, 1u);
    }
    if (tot[3]) atomicOr(&st->overflow, 1u);
  }
}

__device__ void stage_join_probe(const InstDesc& d, InstState* st, const Smem& sm, const uint32_t* bl, uint32_t wmask,
                                 bo_batch_result* res, uint32_t* flag, uint32_t* err) {
  const bo_join_probe_cols p = d.probe;
  const int32_t cl = cap_log2_of(d);
  const uint64_t mask = (1ull << cl) - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int32_t* qf = reinterpret_cast<int32_t*>(sm.b) + warp * 256;
  uint16_t* qo = reinterpret_cast<uint16_t*>(sm.b + kBW * 256 * 4) + warp * 256;
  unsigned __int128* red = reinterpret_cast<unsigned __int128*>(sm.b + kBW * 256 * 6);  // [3][kBW]
  const unsigned long long* slots = d.slots;
  ProbeAcc acc;
  uint32_t c;
  while (next_chunk(&st->cursor[kSJProbe], d.n_chunks[kSJProbe], c)) {
    int64_t lo, hi;
    chunk_range(c, d.unit[kSJProbe], p.n_rows, lo, hi);
    for (int64_t base = lo; base < hi; base += 512) {
      const int64_t r0 = base + lane * 16;
      int32_t fk[16];
      uint32_t valid = 0xffffu;
      if (r0 + 16 <= hi) {
        const int8v f0 = ld_stream_v8(p.fk + r0), f1 = ld_stream_v8(p.fk + r0 + 8);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          fk[k] = f0.v[k];
          fk[8 + k] = f1.v[k];
        }
      } else {
        valid = 0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          fk[k] = 0;
          if (r0 + k < hi) {
            fk[k] = p.fk[r0 + k];
            valid |= 1u << k;
          }
        }
      }
      uint32_t hit = 0;
#pragma unroll
      for (int k = 15; k >= 0; --k) hit = (hit << 1) | bloom_test(bl, wmask, (uint32_t)fk[k]);
      hit &= valid;
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const uint32_t hm = (hit >> (8 * half)) & 0xffu;
        uint32_t total;
        uint32_t pos = warp_exclusive_scan(__popc(hm), total);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          if ((hm >> k) & 1u) {
            qf[pos] = fk[8 * half + k];
            qo[pos] = (uint16_t)(lane * 16 + 8 * half + k);
            ++pos;
          }
        }
        __syncwarp();
        probe_resolve<kProbeResolveB, true>(qf, qo, total, base, slots, mask, kPresizedProbeLimit, p.price, p.discount,
                                            acc);
        __syncwarp();
      }
    }
  }
  if (acc.bad) raise_error(err, acc.bad);
  // Participant totals: warp sums in registers, one pass through shared memory.
  const unsigned __int128 wc = warp_sum_u128(acc.cnt), wt = warp_sum_u128(acc.tsum),
                          wr = warp_sum_u128(acc.rsum);
  if (lane == 0) {
    red[warp] = wc;
    red[kBW + warp] = wt;
    red[2 * kBW + warp] = wr;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned __int128 bc = 0, bt = 0, br = 0;
    for (int w = 0; w < kBW; ++w) {
      bc += red[w];
      bt += red[kBW + w];
      br += red[2 * kBW + w];
    }
    if (bc) atomic_add_i128(&st->acc[0], (__int128)bc);
    if (bt) atomic_add_i128(&st->acc[2], (__int128)bt);
    if (br) atomic_add_i128(&st->acc[4], (__int128)br);
  }
  if (last_tile(&st->ticket, d.n_tiles[kSJProbe], flag) && threadIdx.x == 0) {
    uint32_t fbad = 0;
    const __int128 m = load_i128(&st->acc[0]), t = load_i128(&st->acc[2]), rr = load_i128(&st->acc[4]);
    bo_join_result r;
    r.build_rows = (int64_t)__ldcg(&st->cnt[0]);
    r.distinct_keys = (int64_t)__ldcg(&st->cnt[1]);
    r.match_count = narrow_i64(m, fbad);
    r.sum_trunc = to_bo_i128(t);
    r.sum_exact = to_bo_i128(t * 100 + rr);
    r.capacity_log2 = cl;
    r.overflowed = (int32_t)__ldcg(&st->overflow);
    r.reruns = 0;
    r.mode = 1;
    res->join = r;
    res->kind = BO_BATCH_JOIN;
    res->overflowed = r.overflowed;
    res->reruns = 0;
    if (fbad) raise_error(err, fbad);
  }
}

// Group-by init: one index space of the group slots [0, cap) followed by the
// A-mask words; participant 0 also clears the Bloom filter.
__device__ void stage_gb_init(const InstDesc& d, InstState* st, uint32_t part) {
  const int64_t cap = (int64_t)1 << cap_log2_of(d);
  const int64_t total = cap + d.mask_words;
  if (part == 0)
    for (uint32_t i = threadIdx.x; i < kBloomWords; i += kBB) d.bloom[i] = 0u;
  const int lane = threadIdx.x & 31;
  uint32_t c;
  while (next_chunk(&st->cursor[kSGInit], d.n_chunks[kSGInit], c)) {
    int64_t lo, hi;
    chunk_range(c, d.unit[kSGInit], total, lo, hi);
    for (int64_t i = lo + lane; i < hi; i += 32) {
      if (i < cap) {
        d.slots[i] = kEmptySlot;
        d.mins[i] = 0x7fffffff;
      } else {
        d.amask[i - cap] = 0u;
      }
    }
  }
}

__device__ void stage_gb_cfilter(const InstDesc& d, InstState* st, const Smem& sm, uint32_t (*red)[kBW]) {
  uint32_t* catmask = reinterpret_cast<uint32_t*>(sm.b);
  for (int i = threadIdx.x; i < 2048; i += kBB) catmask[i] = 0u;
  __syncthreads();
  if (threadIdx.x < d.n_cats) atomicOr(&catmask[d.cats[threadIdx.x] >> 5], 1u << (d.cats[threadIdx.x] & 31u));
  __syncthreads();
  const bo_gb_c_cols cc = d.c;
  const int64_t n = cc.n_rows;
  const int32_t year_lo = d.year_lo, year_hi = d.year_hi;
  uint32_t* cbits = d.cbits;
  uint32_t* bloom = d.bloom;
  const int lane = threadIdx.x & 31;
  uint32_t passed = 0, c;
  while (next_chunk(&st->cursor[kSGCFilter], d.n_chunks[kSGCFilter], c)) {
    int64_t w0, w1;
    chunk_range(c, d.unit[kSGCFilter], d.c_words, w0, w1);
    for (int64_t w = w0 + lane; w < w1; w += 32) {
      const int64_t r0 = w * 32;
      uint32_t bits = 0;
      if (r0 + 32 <= n) {
        int8v cat[2];
        cat[0] = ld_stream_v8(cc.category + r0);
        cat[1] = ld_stream_v8(cc.category + r0 + 16);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int8v y = ld_stream_v8(cc.year + r0 + 8 * q);
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
          const uint32_t cv = cc.category[r0 + k];
          const int32_t y = cc.year[r0 + k];
          const bool ok = ((catmask[cv >> 5] >> (cv & 31u)) & 1u) && y >= year_lo && y <= year_hi;
          bits |= (uint32_t)ok << k;
        }
      }
      cbits[w] = bits;
      passed += __popc(bits);
      uint32_t bb = bits;
      while (bb) {
        const int k = __ffs(bb) - 1;
        bb &= bb - 1;
        uint32_t bw, bm;
        bloom_pos((uint32_t)(r0 + k), bw, bm);
        atomicOr(bloom + bw, bm);
      }
    }
  }
  uint32_t tot[4];
  block_counts(passed, 0, 0, 0, red, tot);
  if (threadIdx.x == 0 && tot[0]) atomicAdd(&st->cnt[2], (unsigned long long)tot[0]);
}

__device__ void stage_gb_amask(const InstDesc& d, InstState* st, uint32_t* err) {
  const int32_t* ids = d.a.id;
  const int32_t a_id_max = d.a_id_max;
  uint32_t* amask = d.amask;
  const int lane = threadIdx.x & 31;
  uint32_t bad = 0, c;
  while (next_chunk(&st->cursor[kSGAMask], d.n_chunks[kSGAMask], c)) {
    int64_t lo, hi;
    chunk_range(c, d.unit[kSGAMask], d.a.n_rows, lo, hi);
    for (int64_t i = lo + lane; i < hi; i += 32) {
      const int32_t id = ids[i];
      if (id < 0) continue;  // negative ids are skipped, as by the reference's id masks
      if (id > a_id_max) {
        bad = 1;
        continue;
      }
      atomicOr(amask + (id >> 5), 1u << (id & 31));
    }
  }
  if (bad) raise_error(err, kErrValueRange);
}

__device__ void stage_gb_scan(const InstDesc& d, InstState* st, const Smem& sm, const uint32_t* bl, uint32_t wmask,
                              uint32_t (*red)[kBW]) {
  int32_t* q_c = reinterpret_cast<int32_t*>(sm.b);
  uint32_t* q_row = reinterpret_cast<uint32_t*>(sm.b + kBW * kGbQueueB * 4);
  uint32_t* l_key = reinterpret_cast<uint32_t*>(sm.b + 2 * kBW * kGbQueueB * 4);
  uint32_t* l_cnt = l_key + kGbLocalB;
  int32_t* l_min = reinterpret_cast<int32_t*>(l_cnt + kGbLocalB);
  for (int i = threadIdx.x; i < kGbLocalB; i += kBB) {
    l_key[i] = 0xffffffffu;
    l_cnt[i] = 0u;
    l_min[i] = 0x7fffffff;
  }
  __syncthreads();
  const bo_gb_b_cols b = d.b;
  const int64_t n_c = d.c.n_rows;
  const int32_t* c_year = d.c.year;
  const int32_t a_id_max = d.a_id_max;
  const uint32_t* cbits = d.cbits;
  const uint32_t* amask = d.amask;
  unsigned long long* slots = d.slots;
  int32_t* mins = d.mins;
  const uint64_t mask = (1ull << cap_log2_of(d)) - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int32_t* qc = q_c + warp * kGbQueueB;
  uint32_t* qr = q_row + warp * kGbQueueB;
  uint32_t qn = 0, joined = 0, newkeys = 0, full = 0;
  auto resolve = [&](uint32_t cnt) {
    __syncwarp();
    for (uint32_t i0 = 0; i0 < cnt; i0 += 32 * kGbResolveB) {
      int32_t cc[kGbResolveB], a[kGbResolveB], y[kGbResolveB];
      uint32_t row[kGbResolveB], w[kGbResolveB];
#pragma unroll
      for (int r = 0; r < kGbResolveB; ++r) {
        const uint32_t i = i0 + r * 32 + lane;
        cc[r] = i < cnt ? qc[i] : -1;
        row[r] = i < cnt ? qr[i] : 0u;
        const bool in = (uint32_t)cc[r] < (uint32_t)n_c;
        w[r] = in ? __ldcg(cbits + (cc[r] >> 5)) : 0u;
      }
#pragma unroll
      for (int r = 0; r < kGbResolveB; ++r) {
        const bool pass = (w[r] >> (cc[r] & 31)) & 1u;
        a[r] = pass ? __ldg(b.a_id + row[r]) : -1;
        y[r] = pass ? __ldg(c_year + cc[r]) : 0;
      }
      bool pend[kGbResolveB];
#pragma unroll
      for (int r = 0; r < kGbResolveB; ++r) {
        const bool in_a = a[r] >= 0 && a[r] <= a_id_max;
        const uint32_t m = in_a ? __ldcg(amask + (a[r] >> 5)) : 0u;
        pend[r] = false;
        if (!in_a || !((m >> (a[r] & 31)) & 1u)) continue;
        ++joined;
        const uint32_t h = hash32((uint32_t)a[r]);
        bool done = false;
#pragma unroll 1
        for (int pr = 0; pr < kGbLocalProbesB && !done; ++pr) {
          const int sl = (int)((h + pr) & (kGbLocalB - 1));
          const uint32_t old = atomicCAS(&l_key[sl], 0xffffffffu, (uint32_t)a[r]);
          if (old == 0xffffffffu || old == (uint32_t)a[r]) {
            atomicAdd(&l_cnt[sl], 1u);
            atomicMin(&l_min[sl], y[r]);
            done = true;
          }
        }
        pend[r] = !done;
      }
      unsigned long long got[kGbResolveB];
      uint64_t first[kGbResolveB];
#pragma unroll
      for (int r = 0; r < kGbResolveB; ++r) {
        first[r] = pend[r] ? (hash32((uint32_t)a[r]) & mask) : 0;
        got[r] = pend[r] ? atomicCAS(slots + first[r], kEmptySlot, (unsigned long long)(uint32_t)a[r] << 32) : 0ull;
      }
#pragma unroll
      for (int r = 0; r < kGbResolveB; ++r) {
        if (!pend[r]) continue;
        if (got[r] == kEmptySlot) ++newkeys;
        if (got[r] == kEmptySlot || (uint32_t)(got[r] >> 32) == (uint32_t)a[r]) {
          atomicAdd(slots + first[r], 1ull);
          atomicMin(mins + first[r], y[r]);
        } else if (!gb_global_insert(slots, mins, mask, (uint32_t)a[r], 1u, y[r], newkeys, (first[r] + 1) & mask,
                                       kPresizedProbeLimit)) {
          full = 1;
        }
      }
    }
    __syncwarp();
  };
  uint32_t c;
  while (next_chunk(&st->cursor[kSGScan], d.n_chunks[kSGScan], c)) {
    int64_t lo, hi;
    chunk_range(c, d.unit[kSGScan], b.n_rows, lo, hi);
    for (int64_t base = lo; base < hi; base += 512) {
      const int64_t r0 = base + lane * 16;
      int32_t cid[16];
      uint32_t valid = 0;
      if (r0 + 16 <= hi) {
        const int8v c0 = ld_stream_v8(b.c_id + r0), c1 = ld_stream_v8(b.c_id + r0 + 8);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          cid[k] = c0.v[k];
          cid[8 + k] = c1.v[k];
        }
        valid = 0xffffu;
      } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          cid[k] = -1;
          if (r0 + k < hi) {
            cid[k] = b.c_id[r0 + k];
            valid |= 1u << k;
          }
        }
      }
      uint32_t hit = 0;
#pragma unroll
      for (int k = 15; k >= 0; --k) hit = (hit << 1) | bloom_test(bl, wmask, (uint32_t)cid[k]);
      hit &= valid;
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const uint32_t hm = (hit >> (8 * half)) & 0xffu;
        uint32_t total;
        uint32_t pos = warp_exclusive_scan(__popc(hm), total);
        if (total == 0) continue;
        if (qn + total > kGbQueueB) {
          resolve(qn);
          qn = 0;
        }
        pos += qn;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          if ((hm >> k) & 1u) {
            qc[pos] = cid[8 * half + k];
            qr[pos] = (uint32_t)(r0 + 8 * half + k);
            ++pos;
          }
        }
        qn += total;
        __syncwarp();
        if (qn >= kGbFlushAtB) {
          resolve(qn);
          qn = 0;
        }
      }
    }
  }
  if (qn) resolve(qn);
  __syncthreads();
  for (int i = threadIdx.x; i < kGbLocalB; i += kBB)
    if (l_key[i] != 0xffffffffu)
      if (!gb_global_insert(slots, mins, mask, l_key[i], l_cnt[i], l_min[i], newkeys, ~0ull, kPresizedProbeLimit))
        full = 1;
  uint32_t tot[4];
  block_counts(joined, newkeys, 0, full, red, tot);
  if (threadIdx.x == 0) {
    if (tot[0]) atomicAdd(&st->cnt[0], (unsigned long long)tot[0]);
    if (tot[1]) {
      const unsigned long long before = atomicAdd(&st->cnt[1], (unsigned long long)tot[1]);
      if (before + tot[1] > (mask + 1) - ((mask + 1) >> 3)) atomicOr(&st->overflow, 1u);
    }
    if (tot[3]) atomicOr(&st->overflow, 1u);
  }
}

__device__ void stage_gb_select(const InstDesc& d, InstState* st, uint32_t tile, const Smem& sm, SelCtl* ctl,
                                uint32_t (*red)[kBW], bo_batch_result* res, uint32_t* flag) {
  SelBuf sb;
  sb.keys = reinterpret_cast<unsigned long long*>(sm.b);
  sb.vals = reinterpret_cast<uint32_t*>(sm.b + kSelBuf * 8);
  sb.hist = reinterpret_cast<uint32_t*>(sm.b + kSelBuf * 12);
  sb.ctl = ctl;
  const int k = d.k;
  const int wa = d.wa;
  const unsigned long long cmax = d.cmax;
  int64_t lo, hi;
  const int32_t cl = cap_log2_of(d);
  split_range((int64_t)1 << cl, tile, d.n_tiles[kSGSelect], lo, hi);
  sel_reset(sb);
  uint32_t occ = 0;
  for (int64_t base = lo; base < hi; base += kSelChunk) {
    const unsigned long long bound = ctl->bound;
#pragma unroll
    for (int j = 0; j < kSelChunk / kBB; ++j) {
      const int64_t i = base + j * kBB + threadIdx.x;
      unsigned long long v = i < hi ? __ldcg(d.slots + i) : kEmptySlot;
      const bool ok = v != kEmptySlot;
      occ += ok;
      unsigned long long key = 0;
      uint32_t val = 0;
      if (ok) {
        key = ((cmax - (v & 0xffffffffull)) << wa) | (v >> 32);
        val = (uint32_t)__ldcg(d.mins + i);
      }
      sel_add(sb, ok, key, val, bound);
    }
    __syncthreads();
    const bool full = ctl->n > (uint32_t)kSelChunk;
    __syncthreads();  // the next round's appends change n
    if (full) sel_reduce(sb, k);
  }
  sel_reduce(sb, k);
  // Append this tile's candidates.
  __syncthreads();
  const uint32_t nb = ctl->n;
  if (threadIdx.x == 0) ctl->pos = (uint32_t)atomicAdd(&st->n_cand, (unsigned long long)nb);
  __syncthreads();
  const uint32_t at = ctl->pos;
  for (uint32_t i = threadIdx.x; i < nb; i += kBB) {
    d.cand_keys[at + i] = sb.keys[i];
    d.cand_vals[at + i] = sb.vals[i];
  }
  uint32_t tot[4];
  block_counts(occ, 0, 0, 0, red, tot);
  if (threadIdx.x == 0 && tot[0]) atomicAdd(&st->cnt[3], (unsigned long long)tot[0]);
  if (!last_tile(&st->ticket, d.n_tiles[kSGSelect], flag)) return;
  // Merge every tile's candidates and write the ordered top-k.
  const uint32_t nc = (uint32_t)__ldcg(&st->n_cand);
  sel_reset(sb);
  for (uint32_t c0 = 0; c0 < nc; c0 += kSelChunk) {
    const unsigned long long bound = ctl->bound;
#pragma unroll
    for (int j = 0; j < kSelChunk / kBB; ++j) {
      const uint32_t i = c0 + j * kBB + threadIdx.x;
      const bool ok = i < nc;
      sel_add(sb, ok, ok ? __ldcg(d.cand_keys + i) : 0ull, ok ? __ldcg(d.cand_vals + i) : 0u, bound);
    }
    __syncthreads();
    const bool full = ctl->n > (uint32_t)kSelChunk;
    __syncthreads();
    if (full) sel_reduce(sb, k);
  }
  sel_reduce(sb, k);
  __syncthreads();
  const uint32_t nf = ctl->n;
  const unsigned long long n_groups = __ldcg(&st->cnt[3]);
  if (threadIdx.x < nf) {
    const unsigned long long key = sb.keys[threadIdx.x];
    uint32_t rank = 0;
    for (uint32_t j = 0; j < nf; ++j) rank += sb.keys[j] < key;
    bo_gb_row r;
    r.a_id = (int32_t)(key & ((1ull << wa) - 1ull));
    r.min_year = (int32_t)sb.vals[threadIdx.x];
    r.count = (int64_t)(cmax - (key >> wa));
    res->groupby.rows[rank] = r;
  }
  if (threadIdx.x == 0) {
    bo_gb_result& g = res->groupby;
    g.n_groups = (int64_t)n_groups;
    g.joined_rows = (int64_t)__ldcg(&st->cnt[0]);
    g.c_qualifying = (int64_t)__ldcg(&st->cnt[2]);
    g.exact_distinct = 0;
    g.capacity_log2 = cl;
    g.overflowed = (int32_t)__ldcg(&st->overflow);
    g.reruns = 0;
    g.mode = 1;
    g.n_rows_out = (int32_t)nf;
    g.pad = 0;
    res->kind = BO_BATCH_GROUPBY;
    res->overflowed = g.overflowed;
    res->reruns = 0;
  }
}

// --------------------------------------------------------------- kernel ---
constexpr uint64_t kDepWaitNs = 2000000000ull;  // 2 s bound on a dependency wait

__global__ void __launch_bounds__(kBB, 2)
    batch_kernel(const uint2* __restrict__ items, const uint32_t* __restrict__ plan_hdr,
                 const InstDesc* __restrict__ descs, InstState* states, bo_batch_result* results, uint32_t* ctl_words,
                 uint32_t* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint2 cur;
  __shared__ int32_t bloom_inst;
  __shared__ uint32_t stop;
  __shared__ uint32_t flag;
  __shared__ uint32_t red[4][kBW];
  __shared__ SelCtl selctl;
  uint32_t* head = ctl_words;
  uint32_t* abort_word = ctl_words + 1;
  const uint32_t n_items = plan_hdr[0];  // written by the plan copy before the launch
  const Smem sm{smem, smem + kBloomBytes};
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    bloom_inst = -1;
  }
  __syncthreads();
  uint32_t phase = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      uint32_t s = ld_acquire_u32(abort_word);
      uint2 it = make_uint2(0u, 0u);
      if (!s) {
        const uint32_t i = atomicAdd(head, 1u);
        if (i < n_items) {
          it = items[i];
          const uint32_t inst = it.x & 0xffffu, level = it.x >> 24;
          if (level > 0) {
            const uint32_t need = descs[inst].level_items[level - 1];
            const uint32_t* dc = &states[inst].done[level - 1];
            if (ld_acquire_u32(dc) < need) {
              const uint64_t t0 = global_ns();
              while (ld_acquire_u32(dc) < need) {
                if (ld_acquire_u32(abort_word)) {
                  s = 1;
                  break;
                }
                if (global_ns() - t0 > kDepWaitNs) {
                  raise_error(err, kErrSpinTimeout);
                  atomicExch(abort_word, 1u);
                  s = 1;
                  break;
                }
                __nanosleep(256);
              }
            }
          }
        } else {
          s = 1;
        }
      }
      stop = s;
      cur = it;
    }
    __syncthreads();
    if (stop) break;
    __threadfence();
    const uint2 it = cur;
    const uint32_t inst = it.x & 0xffffu, stage = (it.x >> 16) & 0xffu, level = it.x >> 24, tile = it.y;
    const InstDesc& d = descs[inst];
    InstState* st = states + inst;
    bo_batch_result* res = results + inst;
    // Stages that read a Bloom filter stage it into region A once per block and instance.
    const uint32_t* bl = reinterpret_cast<const uint32_t*>(sm.a);
    uint32_t wmask = kBloomWords - 1u;
    if (stage == kSJProbe || stage == kSGScan) {
      if (bloom_inst != (int32_t)inst) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
          asm volatile("fence.proxy.async.global;" ::: "memory");
          mbar_arrive_expect_tx(&bar, kBloomBytes);
          bulk_copy_g2s(sm.a, d.bloom, kBloomBytes, &bar);
        }
        const bool ok = mbar_wait_bounded(&bar, phase, kWaitLimitNs);
        const bool failed = __syncthreads_or(!ok) != 0;  // block-uniform decision
        phase ^= 1u;
        if (failed) {
          // Never expected: give up the batch (the copy is waited for once
          // more, bounded, so nothing is in flight into shared memory at exit).
          mbar_wait_bounded(&bar, phase ^ 1u, kWaitLimitNs);
          if (threadIdx.x == 0) {
            raise_error(err, kErrSpinTimeout);
            atomicExch(abort_word, 1u);
          }
          break;
        }
        __syncthreads();
        if (threadIdx.x == 0) bloom_inst = (int32_t)inst;
      }
    } else if (stage == kSQ1) {
      if (threadIdx.x == 0) bloom_inst = -1;  // region A is overwritten
    }
    switch (stage) {
      case kSQ1:
        stage_q1(d, st, tile, sm, res, &flag, err);
        break;
      case kSJInit:
        stage_join_init(d, st, tile);
        break;
      case kSJBuild:
        stage_join_build(d, st, sm, red);
        break;
      case kSJProbe:
        stage_join_probe(d, st, sm, bl, wmask, res, &flag, err);
        break;
      case kSGInit:
        stage_gb_init(d, st, tile);
        break;
      case kSGCFilter:
        stage_gb_cfilter(d, st, sm, red);
        break;
      case kSGAMask:
        stage_gb_amask(d, st, err);
        break;
      case kSGScan:
        stage_gb_scan(d, st, sm, bl, wmask, red);
        break;
      case kSGSelect:
        stage_gb_select(d, st, tile, sm, &selctl, red, res, &flag);
        break;
      default:
        break;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(&st->done[level], 1u);
  }
}

// ------------------------------------------------------------------ host ---
int ceil_log2_u64(uint64_t v) {
  int l = 0;
  while ((1ull << l) < v) ++l;
  return l;
}
int bit_len(uint64_t v) {
  int b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return b;
}
// Same presizing rule as the solo presized forms: the smallest power of two
// >= factor * prediction, clamped to [2^10, 2^max_log2].
int32_t presize(float pred, float factor, int32_t max_log2) {
  if (!(pred > 0.0f)) return max_log2;
  const double want = (double)pred * factor;
  int32_t cl = 10;
  while (cl < max_log2 && (double)(1ull << cl) < want) ++cl;
  return cl;
}
int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
// Units per tile for a stage of n units: about n / kTargetTiles, clamped to
// [lo, hi] and rounded up to a multiple of `align`.
int64_t tile_size(int64_t n, int64_t lo, int64_t hi, int64_t align) {
  int64_t t = ceil_div(std::max<int64_t>(n, 1), kTargetTiles);
  t = std::min(std::max(t, lo), std::max(hi, lo));
  return ceil_div(t, align) * align;
}

// A pooled stage of n units: chunks of about n / (kPoolChunksPerWarp x the
// warps of a full GPU) units, clamped to [lo, hi] and a multiple of `align`;
// one participant block per kPoolChunksPerBlock chunks, at most one per worker.
void pool_stage(InstDesc& d, int s, int64_t n, int64_t lo, int64_t hi, int64_t align) {
  int64_t u = ceil_div(std::max<int64_t>(n, 1), kPoolWarps * kPoolChunksPerWarp);
  u = std::min(std::max(u, lo), std::max(hi, lo));
  u = ceil_div(u, align) * align;
  d.unit[s] = u;
  const int64_t chunks = std::max<int64_t>(1, ceil_div(n, u));
  d.n_chunks[s] = (uint32_t)chunks;
  d.n_tiles[s] = (uint32_t)std::min<int64_t>(kPoolMaxParticipants, ceil_div(chunks, kPoolChunksPerBlock));
}

bool cols_ok(std::initializer_list<const void*> ps) {
  for (const void* p : ps)
    if (!p || !aligned32(p)) return false;
  return true;
}

}  // namespace
}  // namespace bo

// A batch owns one device allocation laid out as
//   [plan header | descriptors | items]  written by the plan copy before a launch,
//   [control words + per-instance states] cleared by the graph's memset node,
//   [results]  [table pool]
// and a CUDA graph (memset + persistent kernel) captured once.  Re-planning
// (bo_batch_update) rewrites the plan through a pinned staging buffer and an
// asynchronous copy on the context's stream, so a new set of instances costs
// one copy and one graph launch; it never re-captures or reallocates.
struct bo_batch {
  bo_ctx* ctx = nullptr;
  int32_t max_instances = 0;
  int64_t max_items = 0;
  size_t pool_bytes = 0;
  int n = 0;
  uint32_t n_items = 0;
  std::vector<bo_batch_instance> inst;
  void* dmem = nullptr;
  char* d_plan = nullptr;      // header (256 B) | descriptors | items
  size_t plan_bytes = 0;
  uint32_t* d_ctl = nullptr;   // queue head + abort word (256 B), then the states
  size_t state_bytes = 0;
  bo_batch_result* d_res = nullptr;
  char* d_pool = nullptr;
  char* h_plan[2] = {nullptr, nullptr};  // pinned staging, alternating
  cudaEvent_t plan_done[2] = {nullptr, nullptr};
  int plan_slot = 0;
  bo_batch_result* h_res = nullptr;
  int grid = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool planned = false, launched = false;
};

using namespace bo;

namespace {

constexpr size_t kPlanHdr = 256;

void free_batch(bo_batch* b) {
  if (!b) return;
  if (b->ctx && b->ctx->stream) cudaStreamSynchronize(b->ctx->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  for (int i = 0; i < 2; ++i) {
    if (b->plan_done[i]) cudaEventDestroy(b->plan_done[i]);
    if (b->h_plan[i]) cudaFreeHost(b->h_plan[i]);
  }
  if (b->dmem) cudaFree(b->dmem);
  if (b->h_res) cudaFreeHost(b->h_res);
  delete b;
}

int check_instance(bo_ctx* ctx, const bo_batch_instance& x, int i) {
  switch (x.kind) {
    case BO_BATCH_SCAN_AGG: {
      const bo_fact_cols& c = x.fact;
      if (c.n_rows < 0) return set_error(ctx, BO_ERR_INVALID, "batch[%d]: negative rows", i);
      if (x.n_flag_a < 1 || x.n_flag_b < 1 || x.n_flag_a * x.n_flag_b > BO_Q1_MAX_GROUPS)
        return set_error(ctx, BO_ERR_INVALID, "batch[%d]: group domain %d x %d", i, x.n_flag_a, x.n_flag_b);
      if (c.n_rows > 0 && !cols_ok({c.ship_date, c.quantity, c.ext_price, c.discount, c.tax, c.flag_a, c.flag_b}))
        return set_error(ctx, BO_ERR_INVALID, "batch[%d]: scan column null or not 32-byte aligned", i);
      return BO_OK;
    }
    case BO_BATCH_JOIN: {
      if (x.build.n_rows < 0 || x.probe.n_rows < 0 || x.build.n_rows > 0x7fffffffll)
        return set_error(ctx, BO_ERR_INVALID, "batch[%d]: join row counts", i);
      if (x.build.n_rows > 0 && !cols_ok({x.build.key, x.build.date, x.build.segment}))
        return set_error(ctx, BO_ERR_INVALID, "batch[%d]: build column null or not 32-byte aligned", i);
      if (x.probe.n_rows > 0 && !cols_ok({x.probe.fk, x.probe.price, x.probe.discount}))
        return set_error(ctx, BO_ERR_INVALID, "batch[%d]: probe column null or not 32-byte aligned", i);
      if (x.join.segment_eq < 0 || x.join.segment_eq > 255)
        return set_error(ctx, BO_ERR_INVALID, "batch[%d]: segment_eq outside uint8", i);
      return BO_OK;
    }
    case BO_BATCH_GROUPBY: {
      if (x.a.n_rows < 0 || x.b.n_rows < 0 || x.c.n_rows < 0 || x.c.n_rows > 0x7fffffffll ||
          x.b.n_rows > 0xffffffffll)
        return set_error(ctx, BO_ERR_INVALID, "batch[%d]: group-by row counts", i);
      if (x.a_id_max < 0 || x.k < 0 || x.k > BO_GB_MAX_K || x.n_categories < 0 ||
          x.n_categories > BO_BATCH_MAX_CATS)
        return set_error(ctx, BO_ERR_INVALID, "batch[%d]: group-by parameters", i);
      if (x.b.n_rows > 0 && !cols_ok({x.b.a_id, x.b.c_id}))
        return set_error(ctx, BO_ERR_INVALID, "batch[%d]: B column null or not 32-byte aligned", i);
      if (x.c.n_rows > 0 && !cols_ok({x.c.category, x.c.year}))
        return set_error(ctx, BO_ERR_INVALID, "batch[%d]: C column null or not 32-byte aligned", i);
      if (x.a.n_rows > 0 && !x.a.id) return set_error(ctx, BO_ERR_INVALID, "batch[%d]: A column null", i);
      return BO_OK;
    }
    default:
      return set_error(ctx, BO_ERR_INVALID, "batch[%d]: unknown kind %d", i, x.kind);
  }
}

size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

struct Plan {
  InstDesc d;
  size_t table_bytes;
  uint64_t items;
  double weight;  // bytes the instance streams (orders the queue)
};

// Tile sizes, table sizes and item counts of one instance.
Plan plan_instance(const bo_batch_instance& x) {
  Plan p;
  std::memset(&p.d, 0, sizeof(p.d));
  InstDesc& d = p.d;
  d.kind = x.kind;
  d.pred_dev = x.kind == BO_BATCH_SCAN_AGG ? nullptr : x.predicted_device;
  const int64_t t = x.tile_rows > 0 ? ((int64_t)x.tile_rows + 4095) / 4096 * 4096 : 131072;
  // Default slots per predicted row: the solo presized forms' (join 4,
  // group-by 2.5), so an instance's table matches its solo run's.
  const float factor = x.presize_factor > 0.0f ? x.presize_factor : (x.kind == BO_BATCH_JOIN ? 4.0f : 2.5f);
  d.factor = factor;
  p.table_bytes = 0;
  p.weight = 0.0;
  for (int s = 0; s < kNumStages; ++s) d.unit[s] = 1;
  if (x.kind == BO_BATCH_SCAN_AGG) {
    d.fact = x.fact;
    d.cutoff = x.ship_cutoff;
    d.n_fa = (uint32_t)x.n_flag_a;
    d.n_fb = (uint32_t)x.n_flag_b;
    d.unit[kSQ1] = tile_size(x.fact.n_rows, 16384, t, 1024);
    d.n_chunks[kSQ1] = d.n_tiles[kSQ1] = (uint32_t)std::max<int64_t>(1, ceil_div(x.fact.n_rows, d.unit[kSQ1]));
    p.weight = 38.0 * (double)x.fact.n_rows;
  } else if (x.kind == BO_BATCH_JOIN) {
    d.build = x.build;
    d.probe = x.probe;
    d.date_lt = x.join.date_lt;
    d.seg = (uint32_t)x.join.segment_eq;
    const int32_t max_log2 = std::max(10, ceil_log2_u64((uint64_t)std::max<int64_t>(x.build.n_rows, 1) * 2));
    d.cap_log2 = x.predicted_device ? max_log2 : presize(x.predicted, factor, max_log2);
    const int64_t cap = (int64_t)1 << d.cap_log2;
    pool_stage(d, kSJInit, cap, 2048, 1 << 16, 2048);
    pool_stage(d, kSJBuild, x.build.n_rows, 512, 2 * t, 512);
    pool_stage(d, kSJProbe, x.probe.n_rows, 512, t, 512);
    p.table_bytes = al256(8 * (size_t)cap) + al256(kBloomBytes);
    p.weight = 9.0 * (double)x.build.n_rows + 20.0 * (double)x.probe.n_rows;
  } else {
    d.a = x.a;
    d.b = x.b;
    d.c = x.c;
    for (int i = 0; i < x.n_categories && i < BO_BATCH_MAX_CATS; ++i) d.cats[i] = x.categories[i];
    d.n_cats = x.n_categories;
    d.year_lo = x.year_lo;
    d.year_hi = x.year_hi;
    d.k = x.k;
    d.a_id_max = x.a_id_max;
    d.wa = std::max(1, bit_len((uint64_t)x.a_id_max));
    const int wc = std::max(1, bit_len((uint64_t)x.b.n_rows));
    d.cmax = wc >= 64 ? ~0ull : ((1ull << wc) - 1ull);
    const uint64_t groups_max =
        std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)x.a_id_max + 1, (uint64_t)x.b.n_rows));
    const int32_t max_log2 = std::max(10, bit_len(groups_max * 2 - 1));
    d.cap_log2 = x.predicted_device ? max_log2 : presize(x.predicted, factor, max_log2);
    const int64_t cap = (int64_t)1 << d.cap_log2;
    d.mask_words = ((int64_t)x.a_id_max + 1 + 31) / 32;
    d.c_words = (x.c.n_rows + 31) / 32;
    pool_stage(d, kSGInit, cap + d.mask_words, 2048, 1 << 16, 1024);
    pool_stage(d, kSGCFilter, d.c_words, 32, std::max<int64_t>(32, t / 32), 32);  // bitmap words
    pool_stage(d, kSGAMask, x.a.n_rows, 1024, t, 1024);
    pool_stage(d, kSGScan, x.b.n_rows, 512, t, 512);
    // Select tiles split the slot range of this launch's capacity evenly.
    d.unit[kSGSelect] = tile_size(cap, 2048, 65536, 1024);
    d.n_chunks[kSGSelect] = d.n_tiles[kSGSelect] = (uint32_t)std::max<int64_t>(1, ceil_div(cap, d.unit[kSGSelect]));
    const size_t n_cand = (size_t)d.n_tiles[kSGSelect] * (size_t)std::max(1, x.k);
    p.table_bytes = al256(8 * (size_t)cap) + al256(4 * (size_t)cap) + al256(kBloomBytes) +
                    al256(4 * (size_t)std::max<int64_t>(d.c_words, 1)) + al256(4 * (size_t)d.mask_words) +
                    al256(8 * n_cand) + al256(4 * n_cand);
    p.weight = 8.0 * (double)x.b.n_rows + 6.0 * (double)x.c.n_rows + 4.0 * (double)x.a.n_rows;
  }
  p.items = 0;
  for (int s = 0; s < kNumStages; ++s) {
    if (d.n_tiles[s]) d.level_items[kStageLevel[s]] += d.n_tiles[s];
    p.items += d.n_tiles[s];
  }
  return p;
}

// Points an instance's tables into the pool at `p`.
void carve_tables(InstDesc& d, char* p) {
  const int64_t cap = (int64_t)1 << d.cap_log2;
  if (d.kind == BO_BATCH_JOIN) {
    d.slots = reinterpret_cast<unsigned long long*>(p);
    p += al256(8 * (size_t)cap);
    d.bloom = reinterpret_cast<uint32_t*>(p);
  } else if (d.kind == BO_BATCH_GROUPBY) {
    d.slots = reinterpret_cast<unsigned long long*>(p);
    p += al256(8 * (size_t)cap);
    d.mins = reinterpret_cast<int32_t*>(p);
    p += al256(4 * (size_t)cap);
    d.bloom = reinterpret_cast<uint32_t*>(p);
    p += al256(kBloomBytes);
    d.cbits = reinterpret_cast<uint32_t*>(p);
    p += al256(4 * (size_t)std::max<int64_t>(d.c_words, 1));
    d.amask = reinterpret_cast<uint32_t*>(p);
    p += al256(4 * (size_t)d.mask_words);
    const size_t n_cand = (size_t)d.n_tiles[kSGSelect] * (size_t)std::max(1, d.k);
    d.cand_keys = reinterpret_cast<unsigned long long*>(p);
    p += al256(8 * n_cand);
    d.cand_vals = reinterpret_cast<uint32_t*>(p);
  }
}

int plan_into(bo_ctx* ctx, bo_batch* b, const bo_batch_instance* instances, int32_t n) {
  if (!instances || n < 1 || n > b->max_instances)
    return set_error(ctx, BO_ERR_INVALID, "batch: %d instances (1..%d)", n, b->max_instances);
  for (int i = 0; i < n; ++i) {
    int rc = check_instance(ctx, instances[i], i);
    if (rc) return rc;
  }
  std::vector<Plan> plans(n);
  size_t pool = 0;
  uint64_t n_items = 0;
  for (int i = 0; i < n; ++i) {
    plans[i] = plan_instance(instances[i]);
    pool += plans[i].table_bytes;
    n_items += plans[i].items;
  }
  if (pool > b->pool_bytes)
    return set_error(ctx, BO_ERR_OVERFLOW, "batch: tables need %zu bytes, pool holds %zu", pool, b->pool_bytes);
  if (n_items > (uint64_t)b->max_items)
    return set_error(ctx, BO_ERR_OVERFLOW, "batch: %llu work items, plan holds %lld", (unsigned long long)n_items,
                     (long long)b->max_items);
  // Staging: wait until the copy that last used this buffer has completed.
  const int slot = b->plan_slot;
  b->plan_slot ^= 1;
  BO_CUDA(ctx, cudaEventSynchronize(b->plan_done[slot]));
  char* h = b->h_plan[slot];
  uint32_t* hdr = reinterpret_cast<uint32_t*>(h);
  InstDesc* descs = reinterpret_cast<InstDesc*>(h + kPlanHdr);
  uint2* items = reinterpret_cast<uint2*>(h + kPlanHdr + al256(sizeof(InstDesc) * b->max_instances));
  size_t off = 0;
  for (int i = 0; i < n; ++i) {
    carve_tables(plans[i].d, b->d_pool + off);
    off += plans[i].table_bytes;
    descs[i] = plans[i].d;
  }
  // Work items, level-major; larger instances first inside a level.
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return plans[x].weight > plans[y].weight; });
  uint32_t k = 0;
  for (int level = 0; level < kLevels; ++level)
    for (int i : order)
      for (int s = 0; s < kNumStages; ++s)
        if (kStageLevel[s] == level)
          for (uint32_t t = 0; t < plans[i].d.n_tiles[s]; ++t)
            items[k++] = make_uint2((uint32_t)i | ((uint32_t)s << 16) | ((uint32_t)level << 24), t);
  std::memset(hdr, 0, kPlanHdr);
  hdr[0] = k;
  hdr[1] = (uint32_t)n;
  // One copy of header + descriptors, one of the items.
  BO_CUDA(ctx, cudaMemcpyAsync(b->d_plan, h, kPlanHdr + sizeof(InstDesc) * n, cudaMemcpyHostToDevice, ctx->stream));
  const size_t items_off = kPlanHdr + al256(sizeof(InstDesc) * b->max_instances);
  BO_CUDA(ctx, cudaMemcpyAsync(b->d_plan + items_off, h + items_off, sizeof(uint2) * k, cudaMemcpyHostToDevice,
                               ctx->stream));
  BO_CUDA(ctx, cudaEventRecord(b->plan_done[slot], ctx->stream));
  b->inst.assign(instances, instances + n);
  b->n = n;
  b->n_items = k;
  b->planned = true;
  return BO_OK;
}

int create_batch(bo_ctx* ctx, int32_t max_instances, int64_t max_items, size_t pool_bytes, int32_t workers_per_sm,
                 bo_batch** out) {
  if (!out || max_instances < 1 || max_instances > 4096 || max_items < 1 || max_items > 0x7fffffff)
    return set_error(ctx, BO_ERR_INVALID, "batch: 1..4096 instances and 1..2^31-1 items");
  *out = nullptr;
  bo_batch* b = new bo_batch();
  b->ctx = ctx;
  b->max_instances = max_instances;
  b->max_items = max_items;
  b->pool_bytes = pool_bytes;
  b->plan_bytes = kPlanHdr + al256(sizeof(InstDesc) * max_instances) + al256(sizeof(uint2) * (size_t)max_items);
  b->state_bytes = 256 + sizeof(InstState) * max_instances;
  const size_t off_ctl = al256(b->plan_bytes);
  const size_t off_res = off_ctl + al256(b->state_bytes);
  const size_t off_pool = off_res + al256(sizeof(bo_batch_result) * max_instances);
  const size_t total = off_pool + al256(std::max<size_t>(pool_bytes, 256));
  int rc = BO_OK;
  auto fail = [&](cudaError_t err, const char* what) {
    rc = cuda_fail(ctx, err, what);
    free_batch(b);
    return rc;
  };
  cudaError_t e = cudaMalloc(&b->dmem, total);
  if (e != cudaSuccess) {
    cudaGetLastError();
    free_batch(b);
    return set_error(ctx, BO_ERR_OOM, "batch: cannot allocate %zu bytes", total);
  }
  char* base = static_cast<char*>(b->dmem);
  b->d_plan = base;
  b->d_ctl = reinterpret_cast<uint32_t*>(base + off_ctl);
  b->d_res = reinterpret_cast<bo_batch_result*>(base + off_res);
  b->d_pool = base + off_pool;
  for (int i = 0; i < 2; ++i) {
    if ((e = cudaMallocHost(&b->h_plan[i], b->plan_bytes)) != cudaSuccess) return fail(e, "batch plan staging");
    if ((e = cudaEventCreateWithFlags(&b->plan_done[i], cudaEventDisableTiming)) != cudaSuccess)
      return fail(e, "batch plan events");
  }
  if ((e = cudaMemsetAsync(b->d_res, 0, sizeof(bo_batch_result) * max_instances, ctx->stream)) != cudaSuccess)
    return fail(e, "batch results");
  if ((e = cudaMallocHost(&b->h_res, sizeof(bo_batch_result) * max_instances)) != cudaSuccess)
    return fail(e, "batch host results");
  const void* k = reinterpret_cast<const void*>(&batch_kernel);
  if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes)) != cudaSuccess)
    return fail(e, "batch smem attribute");
  int per_sm = occupancy_blocks(k, kBB, kSmemBytes);
  if (workers_per_sm > 0) per_sm = std::min(per_sm, (int)workers_per_sm);
  b->grid = ctx->num_sms * std::max(1, per_sm);
  // Capture: reset of the queue / states, then the persistent kernel.
  cudaStream_t cs = nullptr;
  if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "batch stream");
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const uint32_t* hdr = reinterpret_cast<const uint32_t*>(b->d_plan);
    const InstDesc* descs = reinterpret_cast<const InstDesc*>(b->d_plan + kPlanHdr);
    const uint2* items = reinterpret_cast<const uint2*>(b->d_plan + kPlanHdr + al256(sizeof(InstDesc) * max_instances));
    cudaMemsetAsync(b->d_ctl, 0, b->state_bytes, cs);
    batch_kernel<<<b->grid, kBB, kSmemBytes, cs>>>(items, hdr, descs, reinterpret_cast<InstState*>(b->d_ctl + 64),
                                                   b->d_res, b->d_ctl, ctx->d_err);
    e = cudaStreamEndCapture(cs, &b->graph);
  }
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) return fail(e, "batch graph capture");
  if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess) return fail(e, "batch graph instantiate");
  if ((e = cudaEventCreate(&b->ev0)) != cudaSuccess || (e = cudaEventCreate(&b->ev1)) != cudaSuccess)
    return fail(e, "batch events");
  *out = b;
  return BO_OK;
}

}  // namespace

extern "C" {

int bo_batch_footprint(const bo_batch_instance* x, int64_t* table_bytes, int64_t* items) {
  if (!x || x->kind < BO_BATCH_SCAN_AGG || x->kind > BO_BATCH_GROUPBY) return BO_ERR_INVALID;
  const Plan p = plan_instance(*x);
  if (table_bytes) *table_bytes = (int64_t)p.table_bytes;
  if (items) *items = (int64_t)p.items;
  return BO_OK;
}

int bo_batch_create_pool(bo_ctx* ctx, int32_t max_instances, int64_t max_items, int64_t pool_bytes,
                         int32_t workers_per_sm, bo_batch** out) {
  BO_CHECK_CTX(ctx);
  if (pool_bytes < 0) return set_error(ctx, BO_ERR_INVALID, "batch: negative pool size");
  return create_batch(ctx, max_instances, max_items, (size_t)pool_bytes, workers_per_sm, out);
}

int bo_batch_create(bo_ctx* ctx, const bo_batch_instance* instances, int32_t n, int32_t workers_per_sm,
                    bo_batch** out) {
  BO_CHECK_CTX(ctx);
  if (!instances || !out || n < 1 || n > 4096) return set_error(ctx, BO_ERR_INVALID, "batch: 1..4096 instances");
  *out = nullptr;
  size_t pool = 0;
  uint64_t items = 0;
  for (int i = 0; i < n; ++i) {
    int rc = check_instance(ctx, instances[i], i);
    if (rc) return rc;
    const Plan p = plan_instance(instances[i]);
    pool += p.table_bytes;
    items += p.items;
  }
  bo_batch* b = nullptr;
  int rc = create_batch(ctx, n, (int64_t)items, pool, workers_per_sm, &b);
  if (rc) return rc;
  if ((rc = plan_into(ctx, b, instances, n))) {
    free_batch(b);
    return rc;
  }
  *out = b;
  return BO_OK;
}

int bo_batch_update(bo_ctx* ctx, bo_batch* b, const bo_batch_instance* instances, int32_t n) {
  BO_CHECK_CTX(ctx);
  if (!b || b->ctx != ctx) return set_error(ctx, BO_ERR_INVALID, "batch: null batch or other context");
  return plan_into(ctx, b, instances, n);
}

int bo_batch_launch(bo_ctx* ctx, bo_batch* b) {
  BO_CHECK_CTX(ctx);
  if (!b || b->ctx != ctx) return set_error(ctx, BO_ERR_INVALID, "batch: null batch or other context");
  if (!b->planned) return set_error(ctx, BO_ERR_INVALID, "batch: no instances planned");
  BO_CUDA(ctx, cudaEventRecord(b->ev0, ctx->stream));
  BO_CUDA(ctx, cudaGraphLaunch(b->exec, ctx->stream));
  BO_CUDA(ctx, cudaEventRecord(b->ev1, ctx->stream));
  ctx->launches += 1;
  b->launched = true;
  return BO_OK;
}

int bo_batch_results(bo_ctx* ctx, bo_batch* b, bo_batch_result* out_host) {
  BO_CHECK_CTX(ctx);
  if (!b || b->ctx != ctx || !out_host) return set_error(ctx, BO_ERR_INVALID, "batch: null argument");
  if (!b->launched) return set_error(ctx, BO_ERR_INVALID, "batch: not launched");
  BO_CUDA(ctx, cudaMemcpyAsync(b->h_res, b->d_res, sizeof(bo_batch_result) * b->n, cudaMemcpyDeviceToHost,
                               ctx->stream));
  uint32_t bits = 0;
  int rc = consume_device_errors(ctx, &bits);
  if (rc) return rc;
  if ((rc = device_error_status(ctx, bits, "batch"))) return rc;
  std::memcpy(out_host, b->h_res, sizeof(bo_batch_result) * b->n);
  // Instances whose presized table overflowed: rerun alone in the exact form.
  for (int i = 0; i < b->n; ++i) {
    bo_batch_result& r = out_host[i];
    if (!r.overflowed) continue;
    const bo_batch_instance& x = b->inst[i];
    if (x.kind == BO_BATCH_JOIN) {
      if ((rc = bo_join_plain(ctx, &x.build, &x.probe, &x.join, &r.join))) return rc;
      r.join.reruns = 1;
      r.join.mode = 1;
    } else if (x.kind == BO_BATCH_GROUPBY) {
      bo_gb_params prm = {x.categories, x.n_categories, x.year_lo, x.year_hi, x.k, x.a_id_max, nullptr};
      if ((rc = bo_groupby_topk_plain(ctx, &x.a, &x.b, &x.c, &prm, &r.groupby))) return rc;
      r.groupby.reruns = 1;
      r.groupby.mode = 1;
    }
    r.reruns = 1;
  }
  return BO_OK;
}

int bo_batch_done(const bo_batch* b) {
  if (!b || !b->launched) return BO_ERR_INVALID;
  const cudaError_t e = cudaEventQuery(b->ev1);
  if (e == cudaSuccess) return 1;
  if (e == cudaErrorNotReady) {
    cudaGetLastError();  // not an error: clear it
    return 0;
  }
  return BO_ERR_CUDA;
}

float bo_batch_last_ms(const bo_batch* b) {
  if (!b || !b->launched) return -1.0f;
  float ms = -1.0f;
  if (cudaEventElapsedTime(&ms, b->ev0, b->ev1) != cudaSuccess) {
    cudaGetLastError();
    return -1.0f;
  }
  return ms;
}

int32_t bo_batch_num_items(const bo_batch* b) { return b ? (int32_t)b->n_items : 0; }

void bo_batch_destroy(bo_batch* b) { free_batch(b); }

}  // extern "C"
