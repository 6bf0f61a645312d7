// Per-row and per-key device helpers shared by the standalone pipeline kernels
// (scan_agg.cu, join.cu, groupby.cu) and the batched persistent kernel
// (batch.cu): the exact fixed-point row arithmetic of the scan / group
// aggregate, the blocked Bloom filter, and the open-addressing table inserts
// and lookups.  Keeping one copy makes the batched and the solo forms compute
// every result with the same code.
#pragma once

#include "common.cuh"

namespace bo {

// ============================================== scan + group aggregate ====
constexpr int kScanBlock = 256;
constexpr int kMaxRowsPerThread = 256;
constexpr int kQ1Sums = 8;  // canonical totals per group, bo_q1_agg order without the doubles

// ------------------------------------------------------------ accumulators --
// Canonical per-group totals (global 128-bit accumulators, index s):
//   0 count  1 qty  2 price  3 disc  4 dp = sum trunc(p*(100-d)/100)
//   5 dpe = sum p*(100-d)  6 ch = sum dp*(100+t)  7 che = sum p*(100-d)*(100+t)
//
// Per-thread partials live in shared memory, one private column per thread
// (layout [group][word][thread], 8-byte words): a row adds into its own group's
// words with a load-add-store, so the update is branch-free, conflict-free
// (a warp touches 32 consecutive words whatever its lanes' groups) and costs a
// handful of instructions instead of one predicated update per group.
// Small sums are bit-packed into one word; kMaxRowsPerThread = 256 bounds
// every field so no packed field can carry into the next.
// The column is private to its thread, so a plain load-add-store suffices (a
// shared-memory atomic would serialise in the atomic unit for nothing).
__device__ __forceinline__ void red_shared_u64(unsigned long long* p, unsigned long long v) {
  *p += v;
}

// Wide layout (0 <= qty, price < 2^31; 0 <= disc, tax <= 100).  With
// p = 100*q + r and m = 100 - d:
//   trunc(p*m/100) = q*m + (r*m)/100 =: T,   p*m = 100*T + rr,  rr = (r*m) % 100
// so the exact forms follow from the reference forms plus the small residues:
//   dpe = 100*sum T + sum rr,   che = 100*sum T*(100+t) + sum rr*(100+t).
// Words per group: 0 qty  1 price  2 T  3 T*(100+t)  4 packed
//   packed = count | disc << 9 | rr << 24 | rr*(100+t) << 39
// (<= 256 rows: count < 2^9, disc sum < 2^15, rr sum < 2^15, rr*(100+t) sum < 2^23).
constexpr int kWideWords = 5;

__device__ __forceinline__ void wide_row(unsigned long long* col, int32_t ship, int32_t cutoff, uint64_t q,
                                         uint64_t p, uint64_t d, uint64_t t, uint32_t fa, uint32_t fb,
                                         uint32_t n_fa, uint32_t n_fb, uint32_t& bad) {
  if (ship > cutoff) return;
  const bool in_range = q < 0x80000000ull && p < 0x80000000ull && d <= 100u && t <= 100u;
  const bool code_ok = fa < n_fa && fb < n_fb;
  if (!(in_range && code_ok)) {
    bad |= (in_range ? 0u : kErrValueRange) | (code_ok ? 0u : kErrBadGroupCode);
    return;
  }
  const uint32_t p32 = (uint32_t)p, m = 100u - (uint32_t)d, tm = 100u + (uint32_t)t;
  const uint32_t pq = p32 / 100u, pr = p32 - pq * 100u;
  const uint32_t rm = pr * m;
  const uint32_t rq = rm / 100u, rr = rm - rq * 100u;
  const uint32_t T = pq * m + rq;
  unsigned long long* w = col + (fa * n_fb + fb) * (kWideWords * kScanBlock);
  red_shared_u64(w, q);
  red_shared_u64(w + kScanBlock, p);
  red_shared_u64(w + 2 * kScanBlock, T);
  red_shared_u64(w + 3 * kScanBlock, (unsigned long long)T * tm);
  red_shared_u64(w + 4 * kScanBlock, 1ull | ((unsigned long long)d << 9) | ((unsigned long long)rr << 24) |
                                         ((unsigned long long)(rr * tm) << 39));
}

// Expands one thread's wide-layout words of group g into the canonical sums.
__device__ __forceinline__ void wide_canon(const unsigned long long* col, int g, int64_t v[kQ1Sums]) {
  const unsigned long long* w = col + g * (kWideWords * kScanBlock);
  const uint64_t pk = w[4 * kScanBlock];
  const int64_t T = (int64_t)w[2 * kScanBlock], TT = (int64_t)w[3 * kScanBlock];
  v[0] = (int64_t)(pk & 0x1ffu);
  v[1] = (int64_t)w[0];
  v[2] = (int64_t)w[kScanBlock];
  v[3] = (int64_t)((pk >> 9) & 0x7fffu);
  v[4] = T;
  v[5] = 100 * T + (int64_t)((pk >> 24) & 0x7fffu);
  v[6] = TT;
  v[7] = 100 * TT + (int64_t)(pk >> 39);
}

// Converts a group's canonical 128-bit totals into the output record.
__device__ __forceinline__ bo_q1_agg q1_record(const __int128 (&t)[8], uint32_t& bad) {
  bo_q1_agg r;
  r.count = narrow_i64(t[0], bad);
  r.sum_qty = narrow_i64(t[1], bad);
  r.sum_base_price = narrow_i64(t[2], bad);
  r.sum_disc = narrow_i64(t[3], bad);
  r.sum_disc_price = narrow_i64(t[4], bad);
  r.sum_disc_price_exact = narrow_i64(t[5], bad);
  r.sum_charge = to_bo_i128(t[6]);
  r.sum_charge_exact = to_bo_i128(t[7]);
  return r;
}

// ======================================================= hash tables =====
constexpr unsigned long long kEmptySlot = ~0ull;
constexpr int kBloomLog2Words = 14;  // 16384 32-bit words = 64 KB = 2^19 bits
constexpr uint32_t kBloomWords = 1u << kBloomLog2Words;
constexpr uint32_t kBloomBytes = kBloomWords * 4u;

// Bloom positions from the key with one multiply (Fibonacci hashing): the word
// from the high bits, two bit positions from the low bits.  Cheap enough for
// every probe row; the table uses the stronger hash32 only for the ~9% that
// pass.
__device__ __forceinline__ void bloom_pos(uint32_t key, uint32_t& word, uint32_t& bits) {
  const uint32_t h2 = key * 0x9E3779B1u;
  word = h2 >> (32 - kBloomLog2Words);
  bits = (1u << (h2 & 31u)) | (1u << ((h2 >> 5) & 31u));
}

// The same test as (word & bits) == bits with two funnel-shift rotates (the
// rotate amount uses the low 5 bits, so no masking): 1 if the key may be in
// the filter.
__device__ __forceinline__ uint32_t bloom_test(const uint32_t* bl, uint32_t wmask, uint32_t key) {
  const uint32_t h2 = key * 0x9E3779B1u;
  const uint32_t x = bl[(h2 >> (32 - kBloomLog2Words)) & wmask];
  return __funnelshift_r(x, x, h2) & __funnelshift_r(x, x, h2 >> 5) & 1u;
}

// Row qualifies on the build side (date < date_lt and segment == seg).
__device__ __forceinline__ bool build_qual(int32_t date, uint32_t seg_byte, int32_t date_lt, uint32_t seg) {
  return date < date_lt && seg_byte == seg;
}

__device__ __forceinline__ uint32_t warp_exclusive_scan(uint32_t v, uint32_t& total) {
  const int lane = threadIdx.x & 31;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

// Inserts one qualifying build key: a new key claims a slot and sets its two
// Bloom bits; a repeated key adds to the multiplicity in the low word.
// Probe-chain bound of presized tables: a table sized from a prediction that
// turns out too low must fail fast (the caller reruns exactly) instead of
// walking ever longer chains; at the loads a presized table is built for
// (<= 0.4 at an exact prediction) chains stay far below it.  Exact-size tables
// pass their capacity as the bound (no limit), and a lookup may stop at the
// bound because a key that needed a longer chain would have flagged overflow.
constexpr uint64_t kPresizedProbeLimit = 256;

__device__ __forceinline__ void join_insert(unsigned long long* slots, uint32_t* bloom, uint64_t mask, int32_t key,
                                            uint32_t& newkeys, bool& full, uint64_t limit) {
  const uint32_t h = hash32((uint32_t)key);
  uint64_t idx = h & mask;
  const unsigned long long mine = ((unsigned long long)(uint32_t)key << 32) | 1ull;
  const uint64_t steps = mask < limit ? mask : limit;
  for (uint64_t step = 0; step <= steps; ++step) {
    const unsigned long long old = atomicCAS(slots + idx, kEmptySlot, mine);
    if (old == kEmptySlot) {
      ++newkeys;
      uint32_t w, bits;
      bloom_pos((uint32_t)key, w, bits);
      atomicOr(bloom + w, bits);
      return;
    }
    if ((uint32_t)(old >> 32) == (uint32_t)key) {
      atomicAdd(slots + idx, 1ull);  // multiplicity lives in the low word
      return;
    }
    idx = (idx + 1) & mask;
  }
  full = true;
}

// With p = 100*q + r and m = 100 - d: trunc(p*m/100) = q*m + (r*m)/100 = T and
// p*m = 100*T + rr, rr = (r*m) % 100 -- exact forms from the reference form.
struct ProbeAcc {
  unsigned long long cnt = 0, rsum = 0;
  unsigned __int128 tsum = 0;
  uint32_t bad = 0;
};

__device__ __forceinline__ void accumulate_match(uint64_t p, uint64_t d, unsigned long long mult, ProbeAcc& a) {
  if (p >= 0x80000000ull || d > 100u) {
    a.bad |= kErrValueRange;
    return;
  }
  const uint32_t m = 100u - (uint32_t)d, pq = (uint32_t)p / 100u, pr = (uint32_t)p - pq * 100u;
  const uint32_t rm = pr * m, rq = rm / 100u, rr = rm - rq * 100u;
  const uint32_t T = pq * m + rq;
  a.cnt += mult;
  a.tsum += (unsigned __int128)((unsigned long long)T * mult);
  a.rsum += (unsigned long long)rr * mult;
}

// Linear-probing continuation for the rare key whose first slot held another key.
// kCoherent reads through L2 only (for a table written earlier in the same launch).
template <bool kCoherent>
static __device__ __noinline__ unsigned long long probe_slow(const unsigned long long* slots, uint64_t mask, uint64_t idx,
                                                      uint32_t key, uint64_t limit) {
  const uint64_t steps = mask < limit ? mask : limit;
  for (uint64_t step = 1; step <= steps; ++step) {
    idx = (idx + 1) & mask;
    const unsigned long long v = kCoherent ? __ldcg(slots + idx) : __ldg(slots + idx);
    if (v == kEmptySlot) return 0;
    if ((uint32_t)(v >> 32) == key) return v & 0xffffffffull;
  }
  return 0;
}

// Resolves a warp's queued probe candidates: keys qf[i] of rows base + qo[i],
// i < total (all lanes call it together).  Each lane takes R entries per round
// and issues their table loads together, then the price / discount loads of
// the matches together, so a warp keeps up to 32 x R lookups in flight instead
// of one dependent chain per lane.  kCoherent reads the table through L2 only
// (for a table written earlier in the same launch).
template <int R, bool kCoherent>
__device__ __forceinline__ void probe_resolve(const int32_t* qf, const uint16_t* qo, uint32_t total, int64_t base,
                                              const unsigned long long* slots, uint64_t mask, uint64_t limit,
                                              const int64_t* price, const int64_t* disc, ProbeAcc& acc) {
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
      v[r] = ok ? (kCoherent ? __ldcg(slots + idx[r]) : __ldg(slots + idx[r])) : kEmptySlot;
    }
    unsigned long long mult[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      mult[r] = 0;
      if (v[r] != kEmptySlot) {
        if ((uint32_t)(v[r] >> 32) == (uint32_t)key[r])
          mult[r] = v[r] & 0xffffffffull;
        else
          mult[r] = probe_slow<kCoherent>(slots, mask, idx[r], (uint32_t)key[r], limit);
      }
    }
    uint64_t pr[R], dc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      pr[r] = mult[r] ? (uint64_t)__ldg(price + row[r]) : 0;
      dc[r] = mult[r] ? (uint64_t)__ldg(disc + row[r]) : 0;
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (mult[r]) accumulate_match(pr[r], dc[r], mult[r], acc);
  }
}

// Group-table insert of a (key, count, min) partial, starting at `start` or at
// the key's hash slot: key << 32 | count words claimed with one CAS, the
// minimum kept beside the slot with atomicMin.
__device__ __forceinline__ bool gb_global_insert(unsigned long long* slots, int32_t* mins, uint64_t mask, uint32_t key,
                                                 uint32_t cnt, int32_t mn, uint32_t& newkeys,
                                                 uint64_t start = ~0ull, uint64_t limit = ~0ull) {
  uint64_t idx = start == ~0ull ? (hash32(key) & mask) : start;
  const unsigned long long claim = (unsigned long long)key << 32;
  const uint64_t steps = mask < limit ? mask : limit;
  for (uint64_t step = 0; step <= steps; ++step) {
    // CAS first: one round trip claims an empty slot or returns its owner.
    unsigned long long v = atomicCAS(slots + idx, kEmptySlot, claim);
    if (v == kEmptySlot) {
      ++newkeys;
      v = claim;
    }
    if ((uint32_t)(v >> 32) == key) {
      atomicAdd(slots + idx, (unsigned long long)cnt);
      atomicMin(mins + idx, mn);
      return true;
    }
    idx = (idx + 1) & mask;
  }
  return false;
}

}  // namespace bo
