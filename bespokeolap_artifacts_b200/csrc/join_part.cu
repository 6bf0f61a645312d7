// Radix-partitioned filtered join + scalar aggregate: the filtered join of
// run_q3 (bespoke_tpch/query_q3.cpp:182-260, restated by join.cu) for build
// sides whose qualifying keys make a table far larger than L2.  The single
// pass (join.cu) then pays a DRAM round trip per probe lookup; here both sides
// are split by the top bits of hash32(key) so that each partition's keys fit
// a table in one SM's shared memory:
//   build   qualifying build rows append their key (one reservation per
//           block tile of 4096 rows),
//           set two bits of a global Bloom filter (L2-resident, sized 16
//           bits per build row), and count into a per-block partition
//           histogram;
//   probe   probe rows whose fk passes the Bloom filter append (fk, row),
//           counted the same way;
//   scatter exclusive scans of the two histograms, then counting scatters
//           group both record arrays by partition;
//   join    one block per partition: its build keys into a shared-memory
//           table (key, multiplicity), its probe records look up there, and
//           matches read price / discount and add the exact fixed-point sums;
//           128-bit totals per block, the last block writes the result.
// A partition with more distinct keys than its table holds (or a longer
// probe chain than the bound) marks the result overflowed and
// bo_join_partitioned reruns the plain single pass; the record arrays take
// the row-count bounds, so they cannot overflow.
#include <algorithm>

#include "common.cuh"
#include "rows.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kJpBlock = 512;
constexpr int kJpSlots = 8192;                      // table slots of one partition
constexpr uint32_t kJpMaxKeys = kJpSlots / 8 * 7;   // fuller counts as overflow
constexpr int kJpProbes = 256;                      // probe-chain bound
constexpr size_t kJpTableSmem = (size_t)kJpSlots * 8;
constexpr int kJpScanBlock = 1024;
constexpr uint32_t kJpEmpty = 0xffffffffu;

struct JpMeta {
  unsigned long long build_rows, distinct;
  unsigned long long acc[6];  // 128-bit match count, sum T, sum rr
  uint32_t b_cursor, p_cursor, overflow, done;
};

// Global blocked Bloom filter of 2^log2w 32-bit words (two bits per key).
struct JpBloom {
  uint32_t* words;
  uint32_t log2w;
  __device__ __forceinline__ void pos(uint32_t key, uint32_t& w, uint32_t& bits) const {
    const uint32_t h = key * 0x9E3779B1u;
    const uint32_t h2 = hash32(key);
    w = log2w ? (h2 >> (32 - log2w)) : 0u;
    bits = (1u << (h & 31u)) | (1u << ((h >> 5) & 31u));
  }
};

__device__ __forceinline__ uint32_t jp_part(uint32_t key, uint32_t shift) {
  return shift >= 32 ? 0u : hash32(key) >> shift;
}

// Rows are read in block tiles of kJpTile (8 consecutive rows per thread,
// 256-bit loads); a tile's records are reserved with one atomic per block (a
// single shared cursor takes one update per 4096 rows, not one per warp).
constexpr int kJpRows = 8;
constexpr int64_t kJpTile = (int64_t)kJpBlock * kJpRows;

// Position of this thread's first record in the tile's reservation of `cnt`
// records per thread (all threads of the block call it).
__device__ __forceinline__ uint32_t jp_block_reserve(uint32_t cnt, uint32_t* cursor, uint32_t* warp_off,
                                                     uint32_t* base) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t wt;
  const uint32_t ex = warp_exclusive_scan(cnt, wt);
  if (lane == 0) warp_off[warp] = wt;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kJpBlock / 32; ++w) {
      const uint32_t x = warp_off[w];
      warp_off[w] = t;
      t += x;
    }
    *base = t ? atomicAdd(cursor, t) : 0u;
  }
  __syncthreads();
  const uint32_t pos = *base + warp_off[warp] + ex;
  __syncthreads();  // warp_off / base are rewritten by the next tile
  return pos;
}

__global__ void __launch_bounds__(kJpBlock) jp_build_kernel(bo_join_build_cols b, int32_t date_lt, uint32_t seg,
                                                            uint32_t shift, uint32_t n_parts, uint32_t* __restrict__ recs,
                                                            JpBloom bloom, uint32_t* __restrict__ counts, JpMeta* meta) {
  extern __shared__ uint32_t hist[];
  __shared__ uint32_t warp_off[kJpBlock / 32];
  __shared__ uint32_t base;
  for (uint32_t i = threadIdx.x; i < n_parts; i += kJpBlock) hist[i] = 0;
  __syncthreads();
  const int64_t n = b.n_rows;
  uint32_t qual = 0;
  for (int64_t t0 = (int64_t)blockIdx.x * kJpTile; t0 < n; t0 += (int64_t)gridDim.x * kJpTile) {
    const int64_t r0 = t0 + (int64_t)threadIdx.x * kJpRows;
    int32_t keys[kJpRows];
    uint32_t take = 0;
    if (r0 + kJpRows <= n) {
      const uint2 sg = ld_stream_v2(b.segment + r0);
      const int8v d = ld_stream_v8(b.date + r0), k = ld_stream_v8(b.key + r0);
#pragma unroll
      for (int j = 0; j < kJpRows; ++j) {
        keys[j] = k.v[j];
        take |= (uint32_t)build_qual(d.v[j], ((j < 4 ? sg.x : sg.y) >> (8 * (j & 3))) & 0xffu, date_lt, seg) << j;
      }
    } else {
#pragma unroll
      for (int j = 0; j < kJpRows; ++j) {
        keys[j] = 0;
        if (r0 + j < n && build_qual(b.date[r0 + j], b.segment[r0 + j], date_lt, seg)) {
          keys[j] = b.key[r0 + j];
          take |= 1u << j;
        }
      }
    }
    qual += __popc(take);
    uint32_t pos = jp_block_reserve(__popc(take), &meta->b_cursor, warp_off, &base);
#pragma unroll
    for (int j = 0; j < kJpRows; ++j) {
      if (!((take >> j) & 1u)) continue;
      const uint32_t key = (uint32_t)keys[j];
      recs[pos++] = key;
      atomicAdd(hist + jp_part(key, shift), 1u);
      uint32_t w, bits;
      bloom.pos(key, w, bits);
      atomicOr(bloom.words + w, bits);
    }
  }
  qual = warp_sum_u32(qual);
  if ((threadIdx.x & 31) == 0 && qual) atomicAdd(&meta->build_rows, (unsigned long long)qual);
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n_parts; i += kJpBlock)
    if (hist[i]) atomicAdd(counts + i, hist[i]);
}

__global__ void __launch_bounds__(kJpBlock) jp_probe_kernel(bo_join_probe_cols p, uint32_t shift, uint32_t n_parts,
                                                            uint2* __restrict__ recs, JpBloom bloom,
                                                            uint32_t* __restrict__ counts, JpMeta* meta) {
  extern __shared__ uint32_t hist[];
  __shared__ uint32_t warp_off[kJpBlock / 32];
  __shared__ uint32_t base;
  for (uint32_t i = threadIdx.x; i < n_parts; i += kJpBlock) hist[i] = 0;
  __syncthreads();
  const int64_t n = p.n_rows;
  for (int64_t t0 = (int64_t)blockIdx.x * kJpTile; t0 < n; t0 += (int64_t)gridDim.x * kJpTile) {
    const int64_t r0 = t0 + (int64_t)threadIdx.x * kJpRows;
    uint32_t fk[kJpRows];
    uint32_t valid = 0;
    if (r0 + kJpRows <= n) {
      const int8v f = ld_stream_v8(p.fk + r0);
#pragma unroll
      for (int j = 0; j < kJpRows; ++j) fk[j] = (uint32_t)f.v[j];
      valid = 0xffu;
    } else {
#pragma unroll
      for (int j = 0; j < kJpRows; ++j) {
        fk[j] = 0;
        if (r0 + j < n) {
          fk[j] = (uint32_t)p.fk[r0 + j];
          valid |= 1u << j;
        }
      }
    }
    uint32_t word[kJpRows], bits[kJpRows];
#pragma unroll
    for (int j = 0; j < kJpRows; ++j) {  // all filter loads issued together
      uint32_t w;
      bloom.pos(fk[j], w, bits[j]);
      word[j] = ((valid >> j) & 1u) ? __ldg(bloom.words + w) : 0u;
    }
    uint32_t take = 0;
#pragma unroll
    for (int j = 0; j < kJpRows; ++j) take |= (uint32_t)((word[j] & bits[j]) == bits[j] && ((valid >> j) & 1u)) << j;
    uint32_t pos = jp_block_reserve(__popc(take), &meta->p_cursor, warp_off, &base);
#pragma unroll
    for (int j = 0; j < kJpRows; ++j) {
      if (!((take >> j) & 1u)) continue;
      recs[pos++] = make_uint2(fk[j], (uint32_t)(r0 + j));
      atomicAdd(hist + jp_part(fk[j], shift), 1u);
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n_parts; i += kJpBlock)
    if (hist[i]) atomicAdd(counts + i, hist[i]);
}

// offsets[i] = records before partition i (offsets[n_parts] = all); fill = offsets.
__global__ void __launch_bounds__(kJpScanBlock) jp_scan_kernel(const uint32_t* __restrict__ counts, uint32_t n_parts,
                                                               uint32_t* __restrict__ offsets,
                                                               uint32_t* __restrict__ fill) {
  __shared__ uint32_t warp_tot[kJpScanBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t per = (n_parts + kJpScanBlock - 1) / kJpScanBlock;
  const uint32_t lo = threadIdx.x * per, hi = min(lo + per, n_parts);
  uint32_t local = 0;
  for (uint32_t i = lo; i < hi; ++i) local += counts[i];
  uint32_t wt;
  const uint32_t wex = warp_exclusive_scan(local, wt);
  if (lane == 0) warp_tot[warp] = wt;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kJpScanBlock / 32; ++w) {
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

// Records -> their partition's range (the lanes of one partition reserve
// their slots with one atomic).
template <class Rec>
__global__ void __launch_bounds__(kJpBlock) jp_scatter_kernel(const Rec* __restrict__ recs, const uint32_t* n_recs,
                                                              uint32_t shift, uint32_t* __restrict__ fill,
                                                              Rec* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const uint32_t n = __ldcg(n_recs);
  const uint32_t warps = gridDim.x * (kJpBlock / 32);
  for (uint32_t i0 = (blockIdx.x * kJpBlock + threadIdx.x) & ~31u; i0 < n; i0 += warps * 32) {
    const uint32_t i = i0 + lane;
    const bool valid = i < n;
    Rec r{};
    uint32_t part = 0xffffffffu;
    if (valid) {
      r = recs[i];
      part = jp_part(*reinterpret_cast<const uint32_t*>(&r), shift);
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, part);
    const int leader = __ffs(peers) - 1;
    uint32_t first = 0;
    if (valid && lane == leader) first = atomicAdd(fill + part, (uint32_t)__popc(peers));
    first = __shfl_sync(0xffffffffu, first, leader);
    if (valid) out[first + __popc(peers & ((1u << lane) - 1u))] = r;
  }
}

__global__ void __launch_bounds__(kJpBlock) jp_join_kernel(const uint32_t* __restrict__ bkeys,
                                                           const uint32_t* __restrict__ boff,
                                                           const uint2* __restrict__ precs,
                                                           const uint32_t* __restrict__ poff, uint32_t n_parts,
                                                           const int64_t* __restrict__ price,
                                                           const int64_t* __restrict__ disc, JpMeta* meta,
                                                           bo_join_result* out, int32_t log2_parts, uint32_t* err) {
  extern __shared__ __align__(16) uint32_t jp_smem[];
  uint32_t* t_key = jp_smem;
  uint32_t* t_cnt = jp_smem + kJpSlots;
  __shared__ uint32_t full_s, used_s;
  __shared__ unsigned __int128 red[kJpBlock + 32];
  ProbeAcc acc;
  uint32_t distinct = 0;
  for (uint32_t p = blockIdx.x; p < n_parts; p += gridDim.x) {
    for (int i = threadIdx.x; i < kJpSlots; i += kJpBlock) {
      t_key[i] = kJpEmpty;
      t_cnt[i] = 0;
    }
    if (threadIdx.x == 0) full_s = used_s = 0;
    __syncthreads();
    for (uint32_t i = boff[p] + threadIdx.x; i < boff[p + 1]; i += kJpBlock) {
      if (*reinterpret_cast<volatile uint32_t*>(&full_s)) break;  // the call reruns: stop early
      const uint32_t key = bkeys[i];
      uint32_t sl = hash32(key) & (kJpSlots - 1);
      bool done = false;
      for (int step = 0; step < kJpProbes && !done; ++step) {
        const uint32_t old = atomicCAS(t_key + sl, kJpEmpty, key);
        if (old == kJpEmpty || old == key) {
          if (old == kJpEmpty) {
            ++distinct;
            if (atomicAdd(&used_s, 1u) + 1u > kJpMaxKeys) full_s = 1;
          }
          atomicAdd(t_cnt + sl, 1u);
          done = true;
        }
        sl = (sl + 1) & (kJpSlots - 1);
      }
      if (!done) full_s = 1;
    }
    __syncthreads();
    if (!full_s) {
      for (uint32_t i = poff[p] + threadIdx.x; i < poff[p + 1]; i += kJpBlock) {
        const uint2 r = precs[i];
        uint32_t sl = hash32(r.x) & (kJpSlots - 1);
        uint32_t mult = 0;
        for (int step = 0; step < kJpProbes; ++step) {
          const uint32_t k = t_key[sl];
          if (k == kJpEmpty) break;
          if (k == r.x) {
            mult = t_cnt[sl];
            break;
          }
          sl = (sl + 1) & (kJpSlots - 1);
        }
        if (mult)
          accumulate_match((uint64_t)__ldg(price + r.y), (uint64_t)__ldg(disc + r.y), (unsigned long long)mult, acc);
      }
    } else if (threadIdx.x == 0) {
      atomicOr(&meta->overflow, 1u);
    }
    __syncthreads();
  }
  if (acc.bad) raise_error(err, acc.bad);
  const unsigned __int128 bc = block_sum_u128(acc.cnt, red);
  const unsigned __int128 bt = block_sum_u128(acc.tsum, red);
  const unsigned __int128 br = block_sum_u128(acc.rsum, red);
  const uint32_t wd = warp_sum_u32(distinct);
  if ((threadIdx.x & 31) == 0 && wd) atomicAdd(&meta->distinct, (unsigned long long)wd);
  if (threadIdx.x == 0) {
    if (bc) atomic_add_i128(&meta->acc[0], (__int128)bc);
    if (bt) atomic_add_i128(&meta->acc[2], (__int128)bt);
    if (br) atomic_add_i128(&meta->acc[4], (__int128)br);
  }
  if (last_block(&meta->done) && threadIdx.x == 0) {
    uint32_t fbad = 0;
    const __int128 m = load_i128(&meta->acc[0]), t = load_i128(&meta->acc[2]), rr = load_i128(&meta->acc[4]);
    bo_join_result res;
    res.build_rows = (int64_t)__ldcg(&meta->build_rows);
    res.distinct_keys = (int64_t)__ldcg(&meta->distinct);
    res.match_count = narrow_i64(m, fbad);
    res.sum_trunc = to_bo_i128(t);
    res.sum_exact = to_bo_i128(t * 100 + rr);
    res.capacity_log2 = log2_parts;
    res.overflowed = (int32_t)__ldcg(&meta->overflow);
    res.reruns = 0;
    res.mode = 2;
    *out = res;
    if (fbad) raise_error(err, fbad);
  }
}

int jp_grid(bo_ctx* ctx, const void* k, int block, size_t smem, int64_t items) {
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(k, block, smem);
  return (int)std::max<int64_t>(1, std::min<int64_t>(resident, (items + block - 1) / block));
}

size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_join_partitioned_device(bo_ctx* ctx, const bo_join_build_cols* b, const bo_join_probe_cols* p,
                                          const bo_join_params* prm, int32_t log2_partitions,
                                          bo_join_result* out_device) {
  BO_CHECK_CTX(ctx);
  if (!b || !p || !prm || !out_device) return set_error(ctx, BO_ERR_INVALID, "join_partitioned: null argument");
  if (log2_partitions < 0 || log2_partitions > BO_JOIN_MAX_LOG2_PARTITIONS)
    return set_error(ctx, BO_ERR_INVALID, "join_partitioned: log2_partitions %d outside [0, %d]", log2_partitions,
                     BO_JOIN_MAX_LOG2_PARTITIONS);
  if (b->n_rows < 0 || p->n_rows < 0 || b->n_rows > 0x7fffffffll || p->n_rows > 0x7fffffffll)
    return set_error(ctx, BO_ERR_INVALID, "join_partitioned: row counts outside [0, 2^31)");
  if ((b->n_rows > 0 && (!b->key || !b->date || !b->segment)) ||
      (p->n_rows > 0 && (!p->fk || !p->price || !p->discount)))
    return set_error(ctx, BO_ERR_INVALID, "join_partitioned: null column");
  if ((b->n_rows > 0 && (!aligned32(b->key) || !aligned32(b->date) || !aligned32(b->segment))) ||
      (p->n_rows > 0 && !aligned32(p->fk)))
    return set_error(ctx, BO_ERR_INVALID, "join_partitioned: columns must be 32-byte aligned");
  if (prm->segment_eq < 0 || prm->segment_eq > 255)
    return set_error(ctx, BO_ERR_INVALID, "join_partitioned: segment_eq %d outside uint8", prm->segment_eq);
  const uint32_t n_parts = 1u << log2_partitions;
  const uint32_t shift = log2_partitions == 0 ? 32u : (uint32_t)(32 - log2_partitions);
  // Bloom filter: 16 bits per build row (at most 64 MiB).
  uint32_t log2w = 11;
  while (log2w < 24 && (1ull << log2w) * 32 < (uint64_t)b->n_rows * 16) ++log2w;
  const size_t nb = (size_t)std::max<int64_t>(b->n_rows, 1), np = (size_t)std::max<int64_t>(p->n_rows, 1);
  const size_t bloom_bytes = al256(4ull << log2w);
  const size_t meta_bytes = al256(sizeof(JpMeta));
  const size_t ctr_bytes = al256(4 * (2 * (size_t)n_parts + 1) * 2 + 4 * (size_t)n_parts * 2);
  const size_t b_bytes = al256(4 * nb), p_bytes = al256(8 * np);
  void* base = nullptr;
  int rc = region(ctx, "join_part", bloom_bytes + meta_bytes + ctr_bytes + 2 * b_bytes + 2 * p_bytes, &base);
  if (rc) return rc;
  char* q = static_cast<char*>(base);
  JpBloom bloom{reinterpret_cast<uint32_t*>(q), log2w};
  JpMeta* meta = reinterpret_cast<JpMeta*>(q + bloom_bytes);
  uint32_t* ctr = reinterpret_cast<uint32_t*>(q + bloom_bytes + meta_bytes);
  uint32_t* b_counts = ctr;                           // n_parts
  uint32_t* p_counts = b_counts + n_parts;            // n_parts
  uint32_t* b_off = p_counts + n_parts;               // n_parts + 1
  uint32_t* p_off = b_off + n_parts + 1;              // n_parts + 1
  uint32_t* b_fill = p_off + n_parts + 1;             // n_parts
  uint32_t* p_fill = b_fill + n_parts;                // n_parts
  char* r = q + bloom_bytes + meta_bytes + ctr_bytes;
  uint32_t* b_recs = reinterpret_cast<uint32_t*>(r);
  uint32_t* b_sorted = reinterpret_cast<uint32_t*>(r + b_bytes);
  uint2* p_recs = reinterpret_cast<uint2*>(r + 2 * b_bytes);
  uint2* p_sorted = reinterpret_cast<uint2*>(r + 2 * b_bytes + p_bytes);
  // The Bloom filter, the counters and the histograms start at zero.
  BO_CUDA(ctx, cudaMemsetAsync(q, 0, bloom_bytes + meta_bytes + 4 * 2 * (size_t)n_parts, ctx->stream));

  static bool ready = false;
  const void* kb = reinterpret_cast<const void*>(&jp_build_kernel);
  const void* kp = reinterpret_cast<const void*>(&jp_probe_kernel);
  const void* kj = reinterpret_cast<const void*>(&jp_join_kernel);
  if (!ready) {
    const int hmax = (int)(4u << BO_JOIN_MAX_LOG2_PARTITIONS);
    BO_CUDA(ctx, cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, hmax));
    BO_CUDA(ctx, cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, hmax));
    BO_CUDA(ctx, cudaFuncSetAttribute(kj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJpTableSmem));
    ready = true;
  }
  const size_t hsmem = 4 * (size_t)n_parts;
  if (b->n_rows > 0) {
    jp_build_kernel<<<jp_grid(ctx, kb, kJpBlock, hsmem, (b->n_rows + kJpRows - 1) / kJpRows), kJpBlock, hsmem,
                      ctx->stream>>>(
        *b, prm->date_lt, (uint32_t)prm->segment_eq, shift, n_parts, b_recs, bloom, b_counts, meta);
    if ((rc = after_launch(ctx, "jp_build_kernel"))) return rc;
  }
  if (p->n_rows > 0) {
    jp_probe_kernel<<<jp_grid(ctx, kp, kJpBlock, hsmem, (p->n_rows + kJpRows - 1) / kJpRows), kJpBlock, hsmem,
                      ctx->stream>>>(
        *p, shift, n_parts, p_recs, bloom, p_counts, meta);
    if ((rc = after_launch(ctx, "jp_probe_kernel"))) return rc;
  }
  jp_scan_kernel<<<1, kJpScanBlock, 0, ctx->stream>>>(b_counts, n_parts, b_off, b_fill);
  if ((rc = after_launch(ctx, "jp_scan_kernel"))) return rc;
  jp_scan_kernel<<<1, kJpScanBlock, 0, ctx->stream>>>(p_counts, n_parts, p_off, p_fill);
  if ((rc = after_launch(ctx, "jp_scan_kernel"))) return rc;
  const int gs = ctx->num_sms * 4;
  jp_scatter_kernel<uint32_t><<<gs, kJpBlock, 0, ctx->stream>>>(b_recs, &meta->b_cursor, shift, b_fill, b_sorted);
  if ((rc = after_launch(ctx, "jp_scatter_kernel"))) return rc;
  jp_scatter_kernel<uint2><<<gs, kJpBlock, 0, ctx->stream>>>(p_recs, &meta->p_cursor, shift, p_fill, p_sorted);
  if ((rc = after_launch(ctx, "jp_scatter_kernel"))) return rc;
  const int gj = (int)std::min<int64_t>(n_parts, (int64_t)ctx->num_sms * occupancy_blocks(kj, kJpBlock, kJpTableSmem));
  jp_join_kernel<<<std::max(gj, 1), kJpBlock, kJpTableSmem, ctx->stream>>>(b_sorted, b_off, p_sorted, p_off, n_parts,
                                                                           p->price, p->discount, meta, out_device,
                                                                           log2_partitions, ctx->d_err);
  return after_launch(ctx, "jp_join_kernel");
}

extern "C" int bo_join_partitioned(bo_ctx* ctx, const bo_join_build_cols* b, const bo_join_probe_cols* p,
                                   const bo_join_params* prm, int32_t log2_partitions, bo_join_result* out_host) {
  BO_CHECK_CTX(ctx);
  if (!out_host) return set_error(ctx, BO_ERR_INVALID, "join_partitioned: null output");
  void* dout = nullptr;
  int rc = region(ctx, "join_part_out", sizeof(bo_join_result), &dout);
  if (rc) return rc;
  if ((rc = bo_join_partitioned_device(ctx, b, p, prm, log2_partitions, static_cast<bo_join_result*>(dout))))
    return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(out_host, dout, sizeof(bo_join_result), cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;  // synchronises the stream
  if ((rc = device_error_status(ctx, bits, "join_partitioned"))) return rc;
  if (out_host->overflowed) {  // a partition's table was too small: the single pass, exactly
    if ((rc = bo_join_plain(ctx, b, p, prm, out_host))) return rc;
    out_host->reruns = 1;
    out_host->mode = 2;
  }
  return BO_OK;
}
