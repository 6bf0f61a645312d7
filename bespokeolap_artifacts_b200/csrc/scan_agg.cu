// Scan + filter + low-cardinality group-by aggregation (Q1 shape) and the
// range-predicate scalar sum (Q6 shape).
//
// Reference loops these kernels replace:
//   run_q1  bespoke_tpch/query_q1.cpp:125-230 (filter shipdate <= cutoff, group by
//           returnflag_linestatus code, int64 sums + __int128 sum_charge_num),
//           finalised at :233-259;
//   run_q6  bespoke_tpch/query_q6.cpp:197-222 (date range, discount band,
//           quantity limit, int64 sum of extendedprice*discount).
//
// Design (HBM-bound streaming scan):
//  * every column is read once with streaming vector loads (no L1 allocation);
//    a thread consumes a chunk of 4 (wide layout) or 8 (storage-plan layout)
//    consecutive rows per iteration; 64-bit columns use 256-bit loads so every
//    load instruction consumes whole 32-byte sectors;
//  * the grid is the resident grid (SMs x blocks/SM) and grows only when a
//    thread would otherwise see more than kMaxRowsPerThread rows, which bounds
//    every per-thread partial (and every bit-packed field) so no sum overflows;
//  * each thread keeps private per-group partials in its own column of shared
//    memory, updated with plain load-add-store (branch-free, bank-conflict-free);
//    a block reduces them through warp shuffles and shared memory into 128-bit
//    totals, and one thread per (group, sum) adds the block's total into
//    global 128-bit accumulators;
//  * the last block to finish (ticket counter) converts the totals into the
//    output records and re-zeroes the accumulators for the next call, so a
//    query is a single launch with no memset.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "rows.cuh"
#include "context.cuh"

namespace bo {

// Storage-plan layout: words per group
//   0 price  1 dp  2 dp*(100+t)  3 p*(100-d)  4 p*(100-d)*(100+t)
//   5 packed = count | disc << 9 | (qty + 32768) << 25
// (<= 256 rows: count < 2^9, disc sum < 2^16, offset qty sum < 2^24).
constexpr int kNarrowWords = 6;

__device__ __forceinline__ void narrow_row(unsigned long long* col, int32_t ship, int32_t cutoff, uint32_t code,
                                           int32_t p, int32_t dprice, uint32_t d, uint32_t t, int32_t q,
                                           uint32_t n_groups, uint32_t& bad) {
  if (ship > cutoff) return;
  if (code >= n_groups) {
    bad |= kErrBadGroupCode;
    return;
  }
  const int32_t tm = 100 + (int32_t)t;
  const int64_t v1 = (int64_t)p * (100 - (int32_t)d);
  unsigned long long* w = col + code * (kNarrowWords * kScanBlock);
  red_shared_u64(w, (unsigned long long)(int64_t)p);
  red_shared_u64(w + kScanBlock, (unsigned long long)(int64_t)dprice);
  red_shared_u64(w + 2 * kScanBlock, (unsigned long long)((int64_t)dprice * tm));
  red_shared_u64(w + 3 * kScanBlock, (unsigned long long)v1);
  red_shared_u64(w + 4 * kScanBlock, (unsigned long long)(v1 * tm));
  red_shared_u64(w + 5 * kScanBlock, 1ull | ((unsigned long long)d << 9) |
                                         ((unsigned long long)(uint32_t)(q + 32768) << 25));
}

__device__ __forceinline__ void narrow_canon(const unsigned long long* col, int g, int64_t v[kQ1Sums]) {
  const unsigned long long* w = col + g * (kNarrowWords * kScanBlock);
  const uint64_t pk = w[5 * kScanBlock];
  const int64_t cnt = (int64_t)(pk & 0x1ffu);
  v[0] = cnt;
  v[1] = (int64_t)(pk >> 25) - 32768 * cnt;
  v[2] = (int64_t)w[0];
  v[3] = (int64_t)((pk >> 9) & 0xffffu);
  v[4] = (int64_t)w[kScanBlock];
  v[5] = (int64_t)w[3 * kScanBlock];
  v[6] = (int64_t)w[2 * kScanBlock];
  v[7] = (int64_t)w[4 * kScanBlock];
}

// Block reduction of the per-thread canonical sums into the global 128-bit
// totals (acc: [group][kQ1Sums][2] words).  A thread's partials come from
// <= 256 rows of < 2^47 each, so warp sums fit int64; the cross-warp sum is
// done in __int128.
template <int NG, bool kWide>
__device__ __forceinline__ void block_flush(const unsigned long long* col, int n_groups, unsigned long long* acc) {
  __shared__ int64_t warp_part[kScanBlock / 32][NG * kQ1Sums];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int g = 0; g < NG; ++g) {
    int64_t v[kQ1Sums];
    if (kWide)
      wide_canon(col, g, v);
    else
      narrow_canon(col, g, v);
#pragma unroll
    for (int s = 0; s < kQ1Sums; ++s) {
      const int64_t r = warp_sum_i64(v[s]);
      if (lane == 0) warp_part[warp][g * kQ1Sums + s] = r;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n_groups * kQ1Sums; i += blockDim.x) {
    __int128 tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += (__int128)warp_part[w][i];
    if (tot != 0) atomic_add_i128(acc + 2 * i, tot);
  }
}

// Converts the totals of group g into the output record and clears them.
__device__ void q1_finalize_group(int g, unsigned long long* acc, bo_q1_agg* out, uint32_t& bad) {
  unsigned long long* a = acc + g * kQ1Sums * 2;
  __int128 t[kQ1Sums];
#pragma unroll
  for (int s = 0; s < kQ1Sums; ++s) t[s] = load_i128(a + 2 * s);
  out[g] = q1_record(t, bad);
#pragma unroll
  for (int s = 0; s < 2 * kQ1Sums; ++s) a[s] = 0ull;
}

template <int NG>
constexpr size_t q1_smem_bytes(bool wide) {
  return sizeof(unsigned long long) * NG * (wide ? kWideWords : kNarrowWords) * kScanBlock;
}

// ------------------------------------------------------------ Q1 kernels ---
template <int NG>
__global__ void __launch_bounds__(kScanBlock) q1_fact_kernel(bo_fact_cols c, int32_t cutoff,
                                                             uint32_t n_fa, uint32_t n_fb,
                                                             unsigned long long* acc, uint32_t* done,
                                                             bo_q1_agg* out, uint32_t* err) {
  extern __shared__ unsigned long long q1_cols[];
  unsigned long long* col = q1_cols + threadIdx.x;
#pragma unroll
  for (int i = 0; i < NG * kWideWords; ++i) col[i * kScanBlock] = 0ull;
  uint32_t bad = 0;
  const int64_t n = c.n_rows;
  const int64_t chunks = n >> 2;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t ch = tid; ch < chunks; ch += stride) {
    const int64_t r = ch << 2;
    const int4 sd = ld_stream_v4(c.ship_date + r);
    const long4v q = ld_stream_v4x64(c.quantity + r), p = ld_stream_v4x64(c.ext_price + r);
    const long4v d = ld_stream_v4x64(c.discount + r), t = ld_stream_v4x64(c.tax + r);
    const uint32_t fa = ld_stream_u32(c.flag_a + r), fb = ld_stream_u32(c.flag_b + r);
    const int32_t ship[4] = {sd.x, sd.y, sd.z, sd.w};
#pragma unroll
    for (int k = 0; k < 4; ++k)
      wide_row(col, ship[k], cutoff, q.v[k], p.v[k], d.v[k], t.v[k], (fa >> (8 * k)) & 0xffu, (fb >> (8 * k)) & 0xffu,
               n_fa, n_fb, bad);
  }
  const int64_t tail = (chunks << 2) + tid;
  if (tail < n) {
    wide_row(col, c.ship_date[tail], cutoff, c.quantity[tail], c.ext_price[tail], c.discount[tail], c.tax[tail],
             c.flag_a[tail], c.flag_b[tail], n_fa, n_fb, bad);
  }
  if (bad) raise_error(err, bad);
  __syncwarp();
  block_flush<NG, true>(col, (int)(n_fa * n_fb), acc);
  if (last_block(done)) {
    uint32_t fbad = 0;
    for (int g = threadIdx.x; g < (int)(n_fa * n_fb); g += blockDim.x) q1_finalize_group(g, acc, out, fbad);
    if (fbad) raise_error(err, fbad);
    if (threadIdx.x == 0) *done = 0u;
  }
}

template <int NG>
__global__ void __launch_bounds__(kScanBlock) q1_lineitem_kernel(bo_lineitem_cols c, int32_t cutoff,
                                                                 uint32_t n_groups,
                                                                 unsigned long long* acc,
                                                                 uint32_t* done, bo_q1_agg* out,
                                                                 uint32_t* err) {
  extern __shared__ unsigned long long q1_cols[];
  unsigned long long* col = q1_cols + threadIdx.x;
#pragma unroll
  for (int i = 0; i < NG * kNarrowWords; ++i) col[i * kScanBlock] = 0ull;
  uint32_t bad = 0;
  const int64_t n = c.n_rows;
  const int64_t chunks = n >> 3;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t ch = tid; ch < chunks; ch += stride) {
    const int64_t r = ch << 3;
    const int4 sd = ld_stream_v4(c.shipdate + r);
    const uint2 gc = ld_stream_v2(c.returnflag_linestatus + r);
    const int8v pr = ld_stream_v8(c.extendedprice + r);
    const int8v dpr = ld_stream_v8(c.discounted_price + r);
    const uint2 dc = ld_stream_v2(c.discount + r);
    const uint2 tx = ld_stream_v2(c.tax + r);
    const int4 qt = ld_stream_v4(c.quantity + r);
    const int32_t ship[8] = {(int16_t)sd.x, sd.x >> 16, (int16_t)sd.y, sd.y >> 16,
                             (int16_t)sd.z, sd.z >> 16, (int16_t)sd.w, sd.w >> 16};
    const int32_t qty[8] = {(int16_t)qt.x, qt.x >> 16, (int16_t)qt.y, qt.y >> 16,
                            (int16_t)qt.z, qt.z >> 16, (int16_t)qt.w, qt.w >> 16};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t sh = (k & 3) * 8;
      const uint32_t code = ((k < 4 ? gc.x : gc.y) >> sh) & 0xffu;
      const uint32_t d = ((k < 4 ? dc.x : dc.y) >> sh) & 0xffu;
      const uint32_t t = ((k < 4 ? tx.x : tx.y) >> sh) & 0xffu;
      narrow_row(col, ship[k], cutoff, code, pr.v[k], dpr.v[k], d, t, qty[k], n_groups, bad);
    }
  }
  const int64_t tail_begin = chunks << 3;
  if (tid < n - tail_begin) {
    const int64_t i = tail_begin + tid;
    narrow_row(col, c.shipdate[i], cutoff, c.returnflag_linestatus[i], c.extendedprice[i], c.discounted_price[i],
               c.discount[i], c.tax[i], c.quantity[i], n_groups, bad);
  }
  if (bad) raise_error(err, bad);
  __syncwarp();
  block_flush<NG, false>(col, (int)n_groups, acc);
  if (last_block(done)) {
    uint32_t fbad = 0;
    for (int g = threadIdx.x; g < (int)n_groups; g += blockDim.x) q1_finalize_group(g, acc, out, fbad);
    if (fbad) raise_error(err, fbad);
    if (threadIdx.x == 0) *done = 0u;
  }
}

// ------------------------------------------------------------- Q6 kernel ---
__global__ void __launch_bounds__(kScanBlock) q6_lineitem_kernel(bo_lineitem_cols c, int32_t start,
                                                                 uint32_t span, int32_t dmin,
                                                                 uint32_t dspan, int32_t qlimit,
                                                                 unsigned long long* acc,
                                                                 uint32_t* done, bo_q6_result* out,
                                                                 uint32_t* err) {
  int64_t rev = 0;
  uint32_t cnt = 0;
  const int64_t n = c.n_rows;
  const int64_t chunks = n >> 3;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // Predicate form of query_q6.cpp:205-219: unsigned range tests.
  auto row = [&](int32_t ship, uint32_t d, int32_t q, int32_t p) {
    const bool keep = (uint32_t)(ship - start) < span && (uint32_t)((int32_t)d - dmin) <= dspan &&
                      q < qlimit;
    if (keep) {
      rev += (int64_t)p * (int64_t)d;
      cnt += 1u;
    }
  };
  for (int64_t ch = tid; ch < chunks; ch += stride) {
    const int64_t r = ch << 3;
    const int4 sd = ld_stream_v4(c.shipdate + r);
    const uint2 dc = ld_stream_v2(c.discount + r);
    const int4 qt = ld_stream_v4(c.quantity + r);
    const int8v pr = ld_stream_v8(c.extendedprice + r);
    const int32_t ship[8] = {(int16_t)sd.x, sd.x >> 16, (int16_t)sd.y, sd.y >> 16,
                             (int16_t)sd.z, sd.z >> 16, (int16_t)sd.w, sd.w >> 16};
    const int32_t qty[8] = {(int16_t)qt.x, qt.x >> 16, (int16_t)qt.y, qt.y >> 16,
                            (int16_t)qt.z, qt.z >> 16, (int16_t)qt.w, qt.w >> 16};
#pragma unroll
    for (int k = 0; k < 8; ++k)
      row(ship[k], ((k < 4 ? dc.x : dc.y) >> ((k & 3) * 8)) & 0xffu, qty[k], pr.v[k]);
  }
  const int64_t tail_begin = chunks << 3;
  if (tid < n - tail_begin) {
    const int64_t i = tail_begin + tid;
    row(c.shipdate[i], c.discount[i], c.quantity[i], c.extendedprice[i]);
  }
  __shared__ int64_t part[kScanBlock / 32][2];
  const int64_t wrev = warp_sum_i64(rev);
  const uint32_t wcnt = warp_sum_u32(cnt);
  if ((threadIdx.x & 31) == 0) {
    part[threadIdx.x >> 5][0] = wrev;
    part[threadIdx.x >> 5][1] = (int64_t)wcnt;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    __int128 tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += (__int128)part[w][threadIdx.x];
    if (tot != 0) atomic_add_i128(acc + 2 * threadIdx.x, tot);
  }
  if (last_block(done)) {
    if (threadIdx.x == 0) {
      uint32_t fbad = 0;
      bo_q6_result r;
      r.revenue_raw = narrow_i64(load_i128(acc), fbad);
      r.count = narrow_i64(load_i128(acc + 2), fbad);
      *out = r;
      acc[0] = acc[1] = acc[2] = acc[3] = 0ull;
      *done = 0u;
      if (fbad) raise_error(err, fbad);
    }
  }
}

// ------------------------------------------------------------------ host ---
namespace {

// Grid for a scan over `chunks` chunks of `rows_per_chunk` rows: the resident
// grid, grown so that no thread sees more than kMaxRowsPerThread rows (its
// chunks plus at most one tail row).
int scan_grid(bo_ctx* ctx, const void* kernel, int64_t chunks, int rows_per_chunk, size_t smem = 0) {
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(kernel, kScanBlock, smem);
  const int64_t cap = (kMaxRowsPerThread - 1) / rows_per_chunk;  // chunks per thread
  const int64_t need = (chunks + cap * kScanBlock - 1) / (cap * kScanBlock);
  int64_t g = resident > need ? resident : need;
  if (g < 1) g = 1;
  if (g > 0x7fffffff) g = 0x7fffffff;
  return (int)g;
}

struct ScanScratch {
  unsigned long long* acc;
  uint32_t* done;
};

int scan_scratch(bo_ctx* ctx, const char* name, ScanScratch* s) {
  void* p = nullptr;
  const size_t acc_bytes = sizeof(unsigned long long) * 2 * kQ1Sums * BO_Q1_MAX_GROUPS;
  int rc = region(ctx, name, acc_bytes + 256, &p);
  if (rc) return rc;
  s->acc = static_cast<unsigned long long*>(p);
  s->done = reinterpret_cast<uint32_t*>(static_cast<char*>(p) + acc_bytes);
  return BO_OK;
}

// Opts a kernel into more than 48 KB of dynamic shared memory (once).
int allow_smem(bo_ctx* ctx, const void* k, size_t bytes) {
  BO_CUDA(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return BO_OK;
}

template <int NG>
int launch_q1_fact(bo_ctx* ctx, const bo_fact_cols& c, int32_t cutoff, uint32_t nfa, uint32_t nfb,
                   const ScanScratch& s, bo_q1_agg* out) {
  const void* k = reinterpret_cast<const void*>(&q1_fact_kernel<NG>);
  constexpr size_t smem = q1_smem_bytes<NG>(true);
  static bool ready = false;
  if (!ready) {
    int rc = allow_smem(ctx, k, smem);
    if (rc) return rc;
    ready = true;
  }
  const int grid = scan_grid(ctx, k, c.n_rows >> 2, 4, smem);
  q1_fact_kernel<NG><<<grid, kScanBlock, smem, ctx->stream>>>(c, cutoff, nfa, nfb, s.acc, s.done, out, ctx->d_err);
  return BO_OK;
}

template <int NG>
int launch_q1_lineitem(bo_ctx* ctx, const bo_lineitem_cols& c, int32_t cutoff, uint32_t ng,
                       const ScanScratch& s, bo_q1_agg* out) {
  const void* k = reinterpret_cast<const void*>(&q1_lineitem_kernel<NG>);
  constexpr size_t smem = q1_smem_bytes<NG>(false);
  static bool ready = false;
  if (!ready) {
    int rc = allow_smem(ctx, k, smem);
    if (rc) return rc;
    ready = true;
  }
  const int grid = scan_grid(ctx, k, c.n_rows >> 3, 8, smem);
  q1_lineitem_kernel<NG><<<grid, kScanBlock, smem, ctx->stream>>>(c, cutoff, ng, s.acc, s.done, out, ctx->d_err);
  return BO_OK;
}

int check_fact(bo_ctx* ctx, const bo_fact_cols* c, int32_t nfa, int32_t nfb) {
  if (!c) return set_error(ctx, BO_ERR_INVALID, "q1: null column set");
  if (c->n_rows < 0) return set_error(ctx, BO_ERR_INVALID, "q1: negative row count");
  // Each factor is bounded before the product is formed, so the product
  // cannot overflow int32 (a wrapped product would pass the group bound).
  if (nfa < 1 || nfb < 1 || nfa > BO_Q1_MAX_GROUPS || nfb > BO_Q1_MAX_GROUPS || nfa * nfb > BO_Q1_MAX_GROUPS)
    return set_error(ctx, BO_ERR_INVALID, "q1: group domain %d x %d exceeds %d groups", nfa, nfb,
                     BO_Q1_MAX_GROUPS);
  if (c->n_rows > 0) {
    const void* ptrs[] = {c->ship_date, c->quantity, c->ext_price, c->discount, c->tax, c->flag_a, c->flag_b};
    for (const void* p : ptrs) {
      if (!p) return set_error(ctx, BO_ERR_INVALID, "q1: null column pointer");
      if (!aligned32(p)) return set_error(ctx, BO_ERR_INVALID, "q1: column pointer not 32-byte aligned");
    }
  }
  return BO_OK;
}

int check_lineitem(bo_ctx* ctx, const bo_lineitem_cols* c, bool need_q1_cols, const char* op) {
  if (!c) return set_error(ctx, BO_ERR_INVALID, "%s: null column set", op);
  if (c->n_rows < 0) return set_error(ctx, BO_ERR_INVALID, "%s: negative row count", op);
  if (c->n_rows == 0) return BO_OK;
  const void* q6[] = {c->shipdate, c->extendedprice, c->discount, c->quantity};
  for (const void* p : q6) {
    if (!p) return set_error(ctx, BO_ERR_INVALID, "%s: null column pointer", op);
    if (!aligned32(p)) return set_error(ctx, BO_ERR_INVALID, "%s: column pointer not 32-byte aligned", op);
  }
  if (need_q1_cols) {
    const void* q1[] = {c->returnflag_linestatus, c->discounted_price, c->tax};
    for (const void* p : q1) {
      if (!p) return set_error(ctx, BO_ERR_INVALID, "%s: null column pointer", op);
      if (!aligned32(p)) return set_error(ctx, BO_ERR_INVALID, "%s: column pointer not 32-byte aligned", op);
    }
  }
  return BO_OK;
}

// Uploads host columns into one device staging region (each column 256-byte
// aligned) and returns the device copies.
template <size_t N>
int stage_columns(bo_ctx* ctx, const char* name, const void* const (&src)[N], const size_t (&bytes)[N],
                  void* (&dst)[N]) {
  size_t total = 0;
  size_t off[N];
  for (size_t i = 0; i < N; ++i) {
    off[i] = total;
    total += (bytes[i] + 255) & ~size_t(255);
  }
  void* base = nullptr;
  int rc = region(ctx, name, total ? total : 256, &base);
  if (rc) return rc;
  for (size_t i = 0; i < N; ++i) {
    dst[i] = static_cast<char*>(base) + off[i];
    if (bytes[i]) BO_CUDA(ctx, cudaMemcpyAsync(dst[i], src[i], bytes[i], cudaMemcpyHostToDevice, ctx->stream));
  }
  return BO_OK;
}

int finish_host(bo_ctx* ctx, void* host_out, const void* dev_out, size_t bytes, const char* op) {
  BO_CUDA(ctx, cudaMemcpyAsync(host_out, dev_out, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  uint32_t bits = 0;
  int rc = consume_device_errors(ctx, &bits);
  if (rc) return rc;
  return device_error_status(ctx, bits, op);
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" {

int bo_q1_fact_device(bo_ctx* ctx, const bo_fact_cols* cols, int32_t ship_cutoff, int32_t n_flag_a,
                      int32_t n_flag_b, bo_q1_agg* out_device) {
  BO_CHECK_CTX(ctx);
  int rc = check_fact(ctx, cols, n_flag_a, n_flag_b);
  if (rc) return rc;
  if (!out_device) return set_error(ctx, BO_ERR_INVALID, "q1: null output");
  ScanScratch s;
  if ((rc = scan_scratch(ctx, "q1_acc", &s))) return rc;
  const int ng = n_flag_a * n_flag_b;
  rc = (ng <= 6) ? launch_q1_fact<6>(ctx, *cols, ship_cutoff, n_flag_a, n_flag_b, s, out_device)
                 : launch_q1_fact<8>(ctx, *cols, ship_cutoff, n_flag_a, n_flag_b, s, out_device);
  if (rc) return rc;
  return after_launch(ctx, "q1_fact_kernel");
}

int bo_q1_fact_host(bo_ctx* ctx, const bo_fact_cols* h, int32_t ship_cutoff, int32_t n_flag_a,
                    int32_t n_flag_b, bo_q1_agg* out_host) {
  BO_CHECK_CTX(ctx);
  if (!h || !out_host) return set_error(ctx, BO_ERR_INVALID, "q1: null argument");
  if (h->n_rows < 0) return set_error(ctx, BO_ERR_INVALID, "q1: negative row count");
  const size_t n = (size_t)h->n_rows;
  const void* const src[7] = {h->ship_date, h->quantity, h->ext_price, h->discount, h->tax, h->flag_a, h->flag_b};
  const size_t bytes[7] = {4 * n, 8 * n, 8 * n, 8 * n, 8 * n, n, n};
  void* dst[7];
  int rc = stage_columns(ctx, "q1_in", src, bytes, dst);
  if (rc) return rc;
  bo_fact_cols d = {static_cast<const int32_t*>(dst[0]), static_cast<const int64_t*>(dst[1]),
                    static_cast<const int64_t*>(dst[2]), static_cast<const int64_t*>(dst[3]),
                    static_cast<const int64_t*>(dst[4]), static_cast<const uint8_t*>(dst[5]),
                    static_cast<const uint8_t*>(dst[6]), h->n_rows};
  void* dout = nullptr;
  if ((rc = region(ctx, "q1_out", sizeof(bo_q1_agg) * BO_Q1_MAX_GROUPS, &dout))) return rc;
  if ((rc = bo_q1_fact_device(ctx, &d, ship_cutoff, n_flag_a, n_flag_b, static_cast<bo_q1_agg*>(dout))))
    return rc;
  return finish_host(ctx, out_host, dout, sizeof(bo_q1_agg) * n_flag_a * n_flag_b, "q1");
}

int bo_q1_lineitem_device(bo_ctx* ctx, const bo_lineitem_cols* cols, int16_t cutoff_offset,
                          int32_t n_groups, bo_q1_agg* out_device) {
  BO_CHECK_CTX(ctx);
  int rc = check_lineitem(ctx, cols, true, "q1");
  if (rc) return rc;
  if (n_groups < 1 || n_groups > BO_Q1_MAX_GROUPS)
    return set_error(ctx, BO_ERR_INVALID, "q1: %d groups outside [1, %d]", n_groups, BO_Q1_MAX_GROUPS);
  if (!out_device) return set_error(ctx, BO_ERR_INVALID, "q1: null output");
  ScanScratch s;
  if ((rc = scan_scratch(ctx, "q1n_acc", &s))) return rc;
  rc = (n_groups <= 6) ? launch_q1_lineitem<6>(ctx, *cols, cutoff_offset, n_groups, s, out_device)
                       : launch_q1_lineitem<8>(ctx, *cols, cutoff_offset, n_groups, s, out_device);
  if (rc) return rc;
  return after_launch(ctx, "q1_lineitem_kernel");
}

int bo_q1_lineitem_host(bo_ctx* ctx, const bo_lineitem_cols* h, int16_t cutoff_offset, int32_t n_groups,
                        bo_q1_agg* out_host) {
  BO_CHECK_CTX(ctx);
  if (!h || !out_host) return set_error(ctx, BO_ERR_INVALID, "q1: null argument");
  if (h->n_rows < 0) return set_error(ctx, BO_ERR_INVALID, "q1: negative row count");
  const size_t n = (size_t)h->n_rows;
  const void* const src[7] = {h->shipdate, h->returnflag_linestatus, h->extendedprice, h->discounted_price,
                              h->discount, h->tax, h->quantity};
  const size_t bytes[7] = {2 * n, n, 4 * n, 4 * n, n, n, 2 * n};
  void* dst[7];
  int rc = stage_columns(ctx, "q1n_in", src, bytes, dst);
  if (rc) return rc;
  bo_lineitem_cols d = {static_cast<const int16_t*>(dst[0]), static_cast<const uint8_t*>(dst[1]),
                        static_cast<const int32_t*>(dst[2]), static_cast<const int32_t*>(dst[3]),
                        static_cast<const uint8_t*>(dst[4]), static_cast<const uint8_t*>(dst[5]),
                        static_cast<const int16_t*>(dst[6]), h->n_rows};
  void* dout = nullptr;
  if ((rc = region(ctx, "q1n_out", sizeof(bo_q1_agg) * BO_Q1_MAX_GROUPS, &dout))) return rc;
  if ((rc = bo_q1_lineitem_device(ctx, &d, cutoff_offset, n_groups, static_cast<bo_q1_agg*>(dout)))) return rc;
  return finish_host(ctx, out_host, dout, sizeof(bo_q1_agg) * n_groups, "q1");
}

int bo_q6_lineitem_device(bo_ctx* ctx, const bo_lineitem_cols* cols, int16_t start_offset, int16_t end_offset,
                          int32_t disc_min, int32_t disc_max, int32_t qty_limit, bo_q6_result* out_device) {
  BO_CHECK_CTX(ctx);
  int rc = check_lineitem(ctx, cols, false, "q6");
  if (rc) return rc;
  if (!out_device) return set_error(ctx, BO_ERR_INVALID, "q6: null output");
  ScanScratch s;
  if ((rc = scan_scratch(ctx, "q6_acc", &s))) return rc;
  const void* k = reinterpret_cast<const void*>(&q6_lineitem_kernel);
  const int grid = scan_grid(ctx, k, cols->n_rows >> 3, 8);
  // Same unsigned-span arithmetic as query_q6.cpp:185-190.
  const uint32_t span = (uint32_t)((int32_t)end_offset - (int32_t)start_offset);
  const uint32_t dspan = (uint32_t)(disc_max - disc_min);
  q6_lineitem_kernel<<<grid, kScanBlock, 0, ctx->stream>>>(*cols, start_offset, span, disc_min, dspan, qty_limit,
                                                            s.acc, s.done, out_device, ctx->d_err);
  return after_launch(ctx, "q6_lineitem_kernel");
}

int bo_q6_lineitem_host(bo_ctx* ctx, const bo_lineitem_cols* h, int16_t start_offset, int16_t end_offset,
                        int32_t disc_min, int32_t disc_max, int32_t qty_limit, bo_q6_result* out_host) {
  BO_CHECK_CTX(ctx);
  if (!h || !out_host) return set_error(ctx, BO_ERR_INVALID, "q6: null argument");
  if (h->n_rows < 0) return set_error(ctx, BO_ERR_INVALID, "q6: negative row count");
  const size_t n = (size_t)h->n_rows;
  const void* const src[4] = {h->shipdate, h->extendedprice, h->discount, h->quantity};
  const size_t bytes[4] = {2 * n, 4 * n, n, 2 * n};
  void* dst[4];
  int rc = stage_columns(ctx, "q6_in", src, bytes, dst);
  if (rc) return rc;
  bo_lineitem_cols d = {};
  d.shipdate = static_cast<const int16_t*>(dst[0]);
  d.extendedprice = static_cast<const int32_t*>(dst[1]);
  d.discount = static_cast<const uint8_t*>(dst[2]);
  d.quantity = static_cast<const int16_t*>(dst[3]);
  d.n_rows = h->n_rows;
  void* dout = nullptr;
  if ((rc = region(ctx, "q6_out", sizeof(bo_q6_result), &dout))) return rc;
  if ((rc = bo_q6_lineitem_device(ctx, &d, start_offset, end_offset, disc_min, disc_max, qty_limit,
                                  static_cast<bo_q6_result*>(dout))))
    return rc;
  return finish_host(ctx, out_host, dout, sizeof(bo_q6_result), "q6");
}

}  // extern "C"

// ===========================================================================
// Allocation-free variant of the wide-layout scan / group-aggregate.
//
// Some callers cannot allocate device memory at the moment they run a query:
// code executing while another component owns every device allocation (a
// host database's memory manager, a plugin sandbox), code running between
// allocations it may not interleave with (inside a stream-ordered region whose
// owner forbids cudaMalloc, or on a path that must not synchronise the device,
// which cudaMalloc / cudaFree can do).  For them this entry point takes no
// context and allocates nothing: the caller passes the stream, the inputs, the
// output and an optional status word; the kernel's scratch (the 128-bit
// per-group totals and the last-block ticket) lives in the file-scope device
// array below, which every GPU that loads this library holds until exit.
//
// Limits and rules (also stated in include/bespoke_gpu.h):
//  * at most BO_Q1_MAX_GROUPS groups (the size the array is laid out for);
//    larger group domains are rejected with BO_ERR_INVALID;
//  * every call shares the array: calls whose work overlaps on the GPU race
//    and must be serialised by the caller (one stream, or events);
//  * each call clears the array on its stream before the kernel, so a call
//    never depends on what an earlier (possibly failed) call left behind;
//  * the first call on a device resolves the array's device address
//    (cudaGetSymbolAddress, with that device current) and sets the kernel's
//    shared-memory attribute; make that first call before any stream capture.
// ===========================================================================
namespace bo {
namespace {

constexpr int kNoAllocAccWords = 2 * kQ1Sums * BO_Q1_MAX_GROUPS;  // 128-bit totals
constexpr int kNoAllocWords = kNoAllocAccWords + 32;               // + ticket counter
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_q1_noalloc_scratch[kNoAllocWords];

std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_ptr[kNoAllocMaxDevices] = {};
int g_noalloc_sms[kNoAllocMaxDevices] = {};

// Per-device set-up, done once with the device current: the array's device
// address (a host-side use of the symbol would be a host stand-in, not a
// device address) and the kernels' dynamic shared-memory opt-in.
int noalloc_setup(int device, unsigned long long** scratch, int* sms) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_q1_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return BO_ERR_CUDA;
    }
    int n_sms = 0;
    if (cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || n_sms < 1)
      return BO_ERR_CUDA;
    if (cudaFuncSetAttribute(reinterpret_cast<const void*>(&q1_fact_kernel<6>),
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)q1_smem_bytes<6>(true)) != cudaSuccess ||
        cudaFuncSetAttribute(reinterpret_cast<const void*>(&q1_fact_kernel<8>),
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)q1_smem_bytes<8>(true)) != cudaSuccess)
      return BO_ERR_CUDA;
    g_noalloc_sms[device] = n_sms;
    g_noalloc_ptr[device] = static_cast<unsigned long long*>(p);
  }
  *scratch = g_noalloc_ptr[device];
  *sms = g_noalloc_sms[device];
  return BO_OK;
}

template <int NG>
int noalloc_launch(const bo_fact_cols& c, int32_t cutoff, uint32_t nfa, uint32_t nfb, unsigned long long* scratch,
                   int sms, bo_q1_agg* out, uint32_t* status, cudaStream_t stream) {
  const void* k = reinterpret_cast<const void*>(&q1_fact_kernel<NG>);
  constexpr size_t smem = q1_smem_bytes<NG>(true);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kScanBlock, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int64_t chunks = c.n_rows >> 2;
  const int64_t cap = (kMaxRowsPerThread - 1) / 4;
  const int64_t need = (chunks + cap * kScanBlock - 1) / (cap * kScanBlock);
  int64_t grid = std::max<int64_t>((int64_t)sms * per_sm, need);
  grid = std::min<int64_t>(std::max<int64_t>(grid, 1), 0x7fffffff);
  q1_fact_kernel<NG><<<(int)grid, kScanBlock, smem, stream>>>(
      c, cutoff, nfa, nfb, scratch, reinterpret_cast<uint32_t*>(scratch + kNoAllocAccWords), out, status);
  return cudaGetLastError() == cudaSuccess ? BO_OK : BO_ERR_CUDA;
}

}  // namespace
}  // namespace bo

extern "C" int bo_q1_fact_device_noalloc(const bo_fact_cols* cols, int32_t ship_cutoff, int32_t n_flag_a,
                                         int32_t n_flag_b, bo_q1_agg* out_device, uint32_t* status_device,
                                         void* cuda_stream) {
  if (!cols || !out_device || cols->n_rows < 0) return BO_ERR_INVALID;
  if (n_flag_a < 1 || n_flag_b < 1 || n_flag_a > BO_Q1_MAX_GROUPS || n_flag_b > BO_Q1_MAX_GROUPS ||
      n_flag_a * n_flag_b > BO_Q1_MAX_GROUPS)
    return BO_ERR_INVALID;
  if (cols->n_rows > 0) {
    const void* ptrs[] = {cols->ship_date, cols->quantity, cols->ext_price, cols->discount,
                          cols->tax,       cols->flag_a,   cols->flag_b};
    for (const void* p : ptrs)
      if (!p || !aligned32(p)) return BO_ERR_INVALID;
  }
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kNoAllocMaxDevices) return BO_ERR_CUDA;
  unsigned long long* scratch = nullptr;
  int sms = 0;
  int rc = noalloc_setup(device, &scratch, &sms);
  if (rc) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  if (cudaMemsetAsync(scratch, 0, sizeof(unsigned long long) * kNoAllocWords, stream) != cudaSuccess)
    return BO_ERR_CUDA;
  const int ng = n_flag_a * n_flag_b;
  return ng <= 6 ? noalloc_launch<6>(*cols, ship_cutoff, n_flag_a, n_flag_b, scratch, sms, out_device,
                                     status_device, stream)
                 : noalloc_launch<8>(*cols, ship_cutoff, n_flag_a, n_flag_b, scratch, sms, out_device,
                                     status_device, stream);
}
