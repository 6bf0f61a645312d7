/*
 * bespoke_gpu.h -- C ABI of the B200 execution engine for the data-parallel hot
 * path of the bespoke OLAP pipelines (scan + filter, join build/probe, group-by
 * aggregation, radix sort / top-k).
 *
 * Conventions
 *  - Plain C: opaque context handle, plain pointers and sizes, int status codes.
 *    No C++ exception and no torch type crosses this boundary.
 *  - Every call returns BO_OK (0) or a negative BO_ERR_* code; the message of
 *    the last failure is available from bo_last_error().
 *  - "_device" entry points take DEVICE pointers and run asynchronously on the
 *    context's stream (capturable in a CUDA graph); "_host" entry points take
 *    HOST pointers, copy inputs in, run, copy results out and synchronise.
 *  - One context per host thread.  All work of a context is ordered on its
 *    stream; a context's scratch state is shared by its calls, so two calls of
 *    the same context must not run concurrently on different streams.
 *  - All aggregates are exact integer / fixed-point arithmetic (int64, with
 *    128-bit totals where the reference uses __int128).
 *
 * Each entry point names the reference interface it replaces
 * (paths relative to the DataManagementLab/BespokeOLAP_Artifacts tree).
 */
#ifndef BESPOKE_GPU_H
#define BESPOKE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
enum {
  BO_OK = 0,
  BO_ERR_INVALID = -1,     /* bad argument (null pointer, misalignment, bad size) */
  BO_ERR_OOM = -2,         /* device or pinned-host allocation failed */
  BO_ERR_OVERFLOW = -3,    /* a presized table/buffer overflowed and retries ran out */
  BO_ERR_TIMEOUT = -4,     /* a bounded device-side wait gave up */
  BO_ERR_CUDA = -5,        /* a CUDA runtime call failed */
  BO_ERR_DATA = -6,        /* input data violates the layout contract (e.g. group code) */
  BO_ERR_UNSUPPORTED = -7  /* no GPU / wrong architecture */
};

typedef struct bo_ctx bo_ctx;

/* Signed 128-bit integer as two 64-bit words (value = hi * 2^64 + lo). */
typedef struct bo_i128 {
  uint64_t lo;
  int64_t hi;
} bo_i128;

/* ------------------------------------------------------------- context ---- */
/* Replaces the process-level set-up the reference's external driver does
 * before query() (bespoke_tpch/query_impl.cpp:142-143: pin to one core). */
int bo_create(bo_ctx** out, int device);
/* Creates the CUDA primary context of `device` -- the cost the first
 * bo_create on it otherwise pays (driver start-up and context creation, on
 * the order of a second) -- and nothing else.  Any thread, any number of
 * times.  No reference counterpart: the drop-in's load() calls it on a
 * background thread so that this start-up overlaps the Parquet reads. */
int bo_device_init(int device);
void bo_destroy(bo_ctx* ctx);
const char* bo_last_error(const bo_ctx* ctx);
/* Use an external CUDA stream (cudaStream_t passed as void*); NULL restores the
 * context's own stream.  The own stream is a blocking stream: it is ordered
 * with the legacy default stream (work a caller issued there, e.g. a PyTorch
 * tensor written on its default stream, completes before the context reads
 * it).  With an external stream the caller orders its inputs itself. */
int bo_set_stream(bo_ctx* ctx, void* cuda_stream);
void* bo_get_stream(const bo_ctx* ctx);
int bo_synchronize(bo_ctx* ctx);
int bo_num_sms(const bo_ctx* ctx);
/* Library version / build string (architecture it was compiled for). */
const char* bo_build_info(void);

/* Device / pinned memory helpers so C and C++ callers need no CUDA headers. */
int bo_device_alloc(bo_ctx* ctx, size_t bytes, void** out);
int bo_device_free(bo_ctx* ctx, void* ptr);
int bo_host_alloc_pinned(bo_ctx* ctx, size_t bytes, void** out);
int bo_host_free_pinned(bo_ctx* ctx, void* ptr);
int bo_copy_h2d(bo_ctx* ctx, void* dst_device, const void* src_host, size_t bytes);
int bo_copy_d2h(bo_ctx* ctx, void* dst_host, const void* src_device, size_t bytes);
/* Kernels launched by this library since the context was created (counted on
 * the host at each launch). */
int64_t bo_launch_count(const bo_ctx* ctx);
/* Waits for the context's stream and turns the device error word (set by the
 * _device entry points' kernels) into a status; clears it. */
int bo_check_errors(bo_ctx* ctx);

/* ===================================================================== Q1 ==
 * Scan + filter + low-cardinality group-by aggregation.
 * Replaces run_q1 (bespoke_tpch/query_q1.cpp:104-283, declared
 * bespoke_tpch/query_q1.hpp:22) and its accumulator Q1Agg (query_q1.cpp:27-34).
 */
#define BO_Q1_MAX_GROUPS 8

/* Per-group exact totals.  Scales: quantity/price x100, discount/tax x100.
 *   sum_disc_price        = sum trunc(price*(100-disc)/100)        (x100)   reference form
 *   sum_charge            = sum trunc(price*(100-disc)/100)*(100+tax) (x1e4) reference sum_charge_num
 *   sum_disc_price_exact  = sum price*(100-disc)                   (x1e4)   exact form
 *   sum_charge_exact      = sum price*(100-disc)*(100+tax)         (x1e6)   exact form
 * In the storage-plan layout "trunc(price*(100-disc)/100)" is the stored
 * discounted_price column (bespoke_tpch/builder_impl.cpp:522-532). */
typedef struct bo_q1_agg {
  int64_t count;
  int64_t sum_qty;
  int64_t sum_base_price;
  int64_t sum_disc;
  int64_t sum_disc_price;
  int64_t sum_disc_price_exact;
  bo_i128 sum_charge;
  bo_i128 sum_charge_exact;
} bo_q1_agg;

/* Fact table in the declared wide layout (38 B/row): ship_date int32 days since
 * 1970-01-01; quantity/ext_price int64 x100; discount/tax int64 x100 in
 * [0,100]; flag_a/flag_b uint8 group flags.  Every column pointer of every
 * entry point in this header must be 32-byte aligned (256-bit vector loads). */
typedef struct bo_fact_cols {
  const int32_t* ship_date;
  const int64_t* quantity;
  const int64_t* ext_price;
  const int64_t* discount;
  const int64_t* tax;
  const uint8_t* flag_a;
  const uint8_t* flag_b;
  int64_t n_rows;
} bo_fact_cols;

/* Lineitem columns in the reference storage-plan layout (15 B/row,
 * bespoke_tpch/builder_impl.hpp:39-66): shipdate int16 offset from 1992-01-01,
 * returnflag_linestatus uint8 code, extendedprice int32 x100, discounted_price
 * int32 x100, discount uint8, tax uint8, quantity int16 x100. */
typedef struct bo_lineitem_cols {
  const int16_t* shipdate;
  const uint8_t* returnflag_linestatus;
  const int32_t* extendedprice;
  const int32_t* discounted_price;
  const uint8_t* discount;
  const uint8_t* tax;
  const int16_t* quantity;
  int64_t n_rows;
} bo_lineitem_cols;

/* Wide layout: keep rows with ship_date <= ship_cutoff; group code =
 * flag_a * n_flag_b + flag_b (must be < n_flag_a*n_flag_b <= 8).
 * out_device receives n_flag_a*n_flag_b bo_q1_agg entries indexed by code. */
int bo_q1_fact_device(bo_ctx* ctx, const bo_fact_cols* cols, int32_t ship_cutoff,
                      int32_t n_flag_a, int32_t n_flag_b, bo_q1_agg* out_device);
int bo_q1_fact_host(bo_ctx* ctx, const bo_fact_cols* host_cols, int32_t ship_cutoff,
                    int32_t n_flag_a, int32_t n_flag_b, bo_q1_agg* out_host);

/* Allocation-free variant of bo_q1_fact_device.  It has no counterpart in the
 * reference.  It is for callers that cannot allocate device memory when they
 * run the query -- a host process whose memory manager owns every device
 * allocation, a plugin that may not call cudaMalloc, or a path that must not
 * risk the device-wide synchronisation cudaMalloc / cudaFree can cause.  It
 * takes no context and allocates nothing: the caller passes the CUDA stream
 * (cudaStream_t as void*, NULL = legacy default stream), the device columns,
 * out_device (n_flag_a*n_flag_b records) and an optional status_device word
 * that the kernel ORs device-side error bits into (the caller zeroes it).
 * With status_device NULL, device-side errors (a value outside its range, a
 * group code outside the domain, a 128-bit total that does not narrow) go
 * unreported: the call still returns BO_OK and the totals may be partial, so
 * pass a status word unless the inputs are known to be valid.
 * The kernel's scratch -- 128-bit per-group totals and a ticket counter --
 * is a fixed file-scope device array of (2*8*BO_Q1_MAX_GROUPS + 32) 64-bit
 * words (1,280 bytes) that every GPU loading this library holds until exit;
 * group domains above BO_Q1_MAX_GROUPS are rejected with BO_ERR_INVALID.
 * Each call clears that array on its stream first; calls that overlap on the
 * GPU share it and race, so the caller must serialise them.  The first call
 * on a device resolves the array's device address and sets a kernel
 * attribute: make it before any stream capture.  That address is kept per
 * device number for the life of the process, so do not call this entry point
 * again on a device after cudaDeviceReset there (the reset unloads the module
 * and the kept address would be stale).  Returns BO_OK, BO_ERR_INVALID
 * or BO_ERR_CUDA (no message: there is no context). */
int bo_q1_fact_device_noalloc(const bo_fact_cols* cols, int32_t ship_cutoff, int32_t n_flag_a,
                              int32_t n_flag_b, bo_q1_agg* out_device, uint32_t* status_device,
                              void* cuda_stream);

/* Storage-plan layout: keep rows with shipdate <= cutoff_offset (the int16
 * cutoff run_q1 derives at query_q1.cpp:111-115); n_groups =
 * returnflag_count * linestatus_count (<= 8). */
int bo_q1_lineitem_device(bo_ctx* ctx, const bo_lineitem_cols* cols, int16_t cutoff_offset,
                          int32_t n_groups, bo_q1_agg* out_device);
int bo_q1_lineitem_host(bo_ctx* ctx, const bo_lineitem_cols* host_cols, int16_t cutoff_offset,
                        int32_t n_groups, bo_q1_agg* out_host);

/* ===================================================================== Q6 ==
 * Range predicates + scalar sum.  Replaces run_q6
 * (bespoke_tpch/query_q6.cpp:155-397, declared query_q6.hpp:15): keeps rows with
 * start <= shipdate < end, disc_min <= discount <= disc_max, quantity < qty_limit
 * and returns revenue_raw = sum extendedprice*discount (x1e4) and the row count. */
typedef struct bo_q6_result {
  int64_t revenue_raw;
  int64_t count;
} bo_q6_result;

int bo_q6_lineitem_device(bo_ctx* ctx, const bo_lineitem_cols* cols, int16_t start_offset,
                          int16_t end_offset, int32_t disc_min, int32_t disc_max,
                          int32_t qty_limit, bo_q6_result* out_device);
int bo_q6_lineitem_host(bo_ctx* ctx, const bo_lineitem_cols* host_cols, int16_t start_offset,
                        int16_t end_offset, int32_t disc_min, int32_t disc_max,
                        int32_t qty_limit, bo_q6_result* out_host);

/* =================================================================== JOIN ==
 * Filtered hash join + scalar aggregate.  Replaces the filtered-join shape of
 * run_q3 (bespoke_tpch/query_q3.cpp:182-260): the reference answers it with a
 * dense cust_in_segment byte map and builder-time CSR ranges
 * (builder_impl.cpp:930-991); here the qualifying build keys go into an
 * open-addressing table in HBM (64-bit slots key<<32 | multiplicity, inserted
 * with atomicCAS) plus a blocked Bloom filter the probe stages into shared
 * memory.  Inner-join semantics: a probe row contributes once per matching
 * build row. */
typedef struct bo_join_build_cols {
  const int32_t* key;
  const int32_t* date;
  const uint8_t* segment;
  int64_t n_rows;
} bo_join_build_cols;

typedef struct bo_join_probe_cols {
  const int32_t* fk;
  const int64_t* price;     /* x100, 0 <= price < 2^31 */
  const int64_t* discount;  /* x100, 0 <= discount <= 100 */
  int64_t n_rows;
} bo_join_probe_cols;

typedef struct bo_join_params {
  int32_t date_lt;     /* build row qualifies when date < date_lt ... */
  int32_t segment_eq;  /* ... and segment == segment_eq */
} bo_join_params;

typedef struct bo_join_result {
  int64_t build_rows;      /* qualifying build rows */
  int64_t distinct_keys;   /* distinct qualifying keys (table occupancy) */
  int64_t match_count;     /* joined rows */
  bo_i128 sum_exact;       /* sum price*(100-discount)            (x1e4) */
  bo_i128 sum_trunc;       /* sum trunc(price*(100-discount)/100) (x100), run_q3's revenue */
  int32_t capacity_log2;   /* table capacity used */
  int32_t overflowed;      /* presized table was too small (result invalid, rerun) */
  int32_t reruns;          /* exact-count reruns performed by the call */
  int32_t mode;            /* 0 plain exact-count, 1 presized from a prediction, 2 radix-partitioned */
} bo_join_result;

/* K7, exact-count pre-pass: number of qualifying build rows (device int64). */
int bo_join_count_device(bo_ctx* ctx, const bo_join_build_cols* build, const bo_join_params* params,
                         int64_t* count_device);
/* Plain form: exact-count pre-pass, one host round trip to size the table,
 * then build and probe.  Synchronises; result on the host. */
int bo_join_plain(bo_ctx* ctx, const bo_join_build_cols* build, const bo_join_probe_cols* probe,
                  const bo_join_params* params, bo_join_result* out_host);
/* Presized form, fully asynchronous (no host round trip, capturable in a CUDA
 * graph): the table is sized on the device from predicted_rows_device (one
 * float, the predicted number of qualifying build rows, e.g. an MLP output
 * written by bo_mlp_infer_device).  out_device->overflowed reports a table
 * that turned out too small. */
int bo_join_presized_device(bo_ctx* ctx, const bo_join_build_cols* build, const bo_join_probe_cols* probe,
                            const bo_join_params* params, const float* predicted_rows_device,
                            bo_join_result* out_device);
/* Presized form with the exact fallback: runs bo_join_presized_device,
 * synchronises once, and reruns the plain form if the table overflowed, so
 * the answer never depends on the prediction. */
int bo_join_presized(bo_ctx* ctx, const bo_join_build_cols* build, const bo_join_probe_cols* probe,
                     const bo_join_params* params, const float* predicted_rows_device,
                     bo_join_result* out_host);
/* Probes the table left by this context's most recent join build with another
 * probe batch (asynchronous; the build side is reused).  Used to time the
 * probe kernel alone and to join several probe batches against one build. */
int bo_join_probe_device(bo_ctx* ctx, const bo_join_probe_cols* probe, bo_join_result* out_device);
/* Host buffers in, result out: copies both sides to the device inside the
 * call, then runs the plain (mode 0) or presized (mode 1, prediction given as
 * a host float) form. */
int bo_join_host(bo_ctx* ctx, const bo_join_build_cols* build_host, const bo_join_probe_cols* probe_host,
                 const bo_join_params* params, int32_t mode, float predicted_rows, bo_join_result* out_host);

/* Radix-partitioned form (2^log2_partitions partitions, 0..BO_JOIN_MAX_LOG2_PARTITIONS)
 * for qualifying build keys far beyond L2: qualifying build keys and the probe
 * rows that pass a global Bloom filter of them are split by the top bits of
 * their key's hash (record arrays sized by the row counts, counting scatter),
 * then one block per partition joins the partition in a shared-memory table
 * (8192 slots), so no lookup leaves the SM.  The caller picks the fan-out
 * (learned.JoinSizer.fanout on the predicted qualifying rows: a single pass
 * while its table stays in L2, else partitions of about 4096 keys).  A
 * partition with more distinct keys than its table holds sets overflowed;
 * bo_join_partitioned then reruns the plain single pass (reruns = 1). */
#define BO_JOIN_MAX_LOG2_PARTITIONS 14
int bo_join_partitioned_device(bo_ctx* ctx, const bo_join_build_cols* build, const bo_join_probe_cols* probe,
                               const bo_join_params* params, int32_t log2_partitions, bo_join_result* out_device);
int bo_join_partitioned(bo_ctx* ctx, const bo_join_build_cols* build, const bo_join_probe_cols* probe,
                        const bo_join_params* params, int32_t log2_partitions, bo_join_result* out_host);

/* Shared joins: n_queries (1..BO_JOIN_MULTI_MAX) filtered joins of the same
 * build and probe tables that differ only in their predicate constants, in
 * one count, one build and one probe pass (the table maps a key to the mask
 * of the queries it qualifies for).  out[i] is the result bo_join_plain
 * returns for params[i] (capacity_log2 is the shared table's).  No reference
 * counterpart: it serves concurrent requests (the reference runs one query
 * per call, bespoke_tpch/query_impl.cpp:159-388).  A key that qualifies
 * through two build rows cannot carry per-query multiplicities in the shared
 * table: then every record has overflowed = 1 and the queries must run alone
 * -- bo_join_multi_host does that itself (reruns = 1).  The _device form is
 * asynchronous (out_device: n_queries records), the _host form synchronises. */
#define BO_JOIN_MULTI_MAX 32
int bo_join_multi_device(bo_ctx* ctx, const bo_join_build_cols* build, const bo_join_probe_cols* probe,
                         const bo_join_params* params_host, int32_t n_queries, bo_join_result* out_device);
int bo_join_multi_host(bo_ctx* ctx, const bo_join_build_cols* build, const bo_join_probe_cols* probe,
                       const bo_join_params* params_host, int32_t n_queries, bo_join_result* out_host);

/* Streamed form for inputs in pinned host memory (bo_host_alloc_pinned or
 * cudaHostRegister'd): only the columns every row needs cross PCIe as copies
 * (build date and segment, probe fk, the latter in 1M-row chunks overlapped
 * with the probe of the previous chunks); the build keys of qualifying rows
 * are read in place by the build kernel (zero-copy).  The price / discount of
 * matching probe rows are, by default, gathered by host threads: the probe
 * lists the matching rows of each chunk in pinned host memory, the context's
 * threads copy those rows' price and discount into contiguous records while
 * later chunks are copied and probed, and one bulk copy per chunk feeds a
 * summing kernel (bo_set_host_threads).  With 0 host threads the probe reads
 * them in place instead.  pred_device = NULL runs the exact-count form;
 * otherwise the table is presized from the device prediction and rerun
 * exactly on overflow.  Inputs must stay valid until the call (or, for the
 * _async form, bo_synchronize) returns. */
int bo_join_stream_host(bo_ctx* ctx, const bo_join_build_cols* build_host, const bo_join_probe_cols* probe_host,
                        const bo_join_params* prm, const float* pred_device, bo_join_result* out_host);
/* The presized streamed form without waiting: the result lands in out_pinned
 * (pinned host memory) once the context's stream reaches it (bo_synchronize /
 * bo_check_errors).  Consecutive calls overlap one query's copies with the
 * previous query's kernels (two buffer sets).  A result with `overflowed` set
 * is invalid: rerun that query with bo_join_stream_host. */
int bo_join_stream_host_async(bo_ctx* ctx, const bo_join_build_cols* build_host, const bo_join_probe_cols* probe_host,
                              const bo_join_params* prm, const float* pred_device, bo_join_result* out_pinned);
/* Host threads the streamed join uses to gather the payload of matching probe
 * rows: threads < 0 chooses from the machine (half its hardware threads, at
 * most 8; the default), 0 reads the payload in place over PCIe instead, at
 * most 256.  Waits for queued streamed joins before it takes effect.
 * bo_host_threads returns the count in effect. */
int bo_set_host_threads(bo_ctx* ctx, int32_t threads);
int bo_host_threads(const bo_ctx* ctx);

/* =============================================================== GROUP-BY ==
 * Skewed three-way join + high-cardinality group-by + ordered top-k.  Restates
 * the dense-mask / per-id count pattern of run_q1a
 * (bespoke_ceb/query_q1a.cpp:503-601), the min aggregate of run_q10a
 * (bespoke_ceb/query_q10a.cpp:843-856) and the (count desc, id asc) ordering of
 * radix_sort_groups (bespoke_tpch/query_q10.cpp:318-372):
 *   C row (c_id = row index) qualifies when category is in the set and
 *   year_lo <= year <= year_hi; B row (a_id, c_id) joins when 0 <= c_id <
 *   n_C, C[c_id] qualifies and a_id is an id of A; group by a_id: count,
 *   min(C.year); order by count desc, a_id asc; first k. */
#define BO_GB_MAX_K 64
typedef struct bo_gb_a_cols {
  const int32_t* id;
  int64_t n_rows;
} bo_gb_a_cols;
typedef struct bo_gb_b_cols {
  const int32_t* a_id;
  const int32_t* c_id;
  int64_t n_rows;
} bo_gb_b_cols;
typedef struct bo_gb_c_cols {
  const uint16_t* category;
  const int32_t* year;
  int64_t n_rows;
} bo_gb_c_cols;
typedef struct bo_gb_params {
  const uint16_t* categories;  /* host array, at most 64 values */
  int32_t n_categories;
  int32_t year_lo, year_hi;
  int32_t k;                   /* <= BO_GB_MAX_K */
  int32_t a_id_max;            /* every id of A lies in [0, a_id_max] (negative ids are skipped) */
  const uint32_t* a_mask;      /* optional device bitmap of A's ids over [0, a_id_max], built once per
                                  table by bo_groupby_a_mask_device; NULL builds it inside the call */
} bo_gb_params;
typedef struct bo_gb_row {
  int32_t a_id;
  int32_t min_year;
  int64_t count;
} bo_gb_row;
typedef struct bo_gb_result {
  int64_t n_groups;        /* groups (distinct qualifying a_id) */
  int64_t joined_rows;     /* B rows that joined */
  int64_t c_qualifying;    /* qualifying C rows */
  int64_t exact_distinct;  /* plain form: the exact pre-pass count */
  int32_t capacity_log2;
  int32_t overflowed;      /* presized table too small (result invalid, rerun) */
  int32_t reruns;
  int32_t mode;            /* 0 plain exact-count, 1 presized, 2 radix-partitioned */
  int32_t n_rows_out;      /* min(k, n_groups) */
  int32_t pad;
  bo_gb_row rows[BO_GB_MAX_K];
} bo_gb_result;

/* Plain form: exact distinct-group pre-pass (a full scan of B), one host
 * round trip to size the group table, then the aggregation scan, compaction,
 * onesweep sort and top-k.  Synchronises. */
int bo_groupby_topk_plain(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b, const bo_gb_c_cols* c,
                          const bo_gb_params* params, bo_gb_result* out_host);
/* Presized form, asynchronous: the group table is sized on the device from a
 * predicted group count (device float, e.g. an MLP output); one scan of B. */
int bo_groupby_topk_presized_device(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b,
                                    const bo_gb_c_cols* c, const bo_gb_params* params,
                                    const float* predicted_groups_device, bo_gb_result* out_device);
/* Presized form with the exact fallback (rerun in the plain form on overflow). */
int bo_groupby_topk_presized(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b, const bo_gb_c_cols* c,
                             const bo_gb_params* params, const float* predicted_groups_device,
                             bo_gb_result* out_host);
/* Radix-partitioned form (2^log2_partitions partitions, 0..BO_GB_MAX_LOG2_PARTITIONS):
 * the scan of B writes each surviving row -- or, for keys the block
 * pre-aggregated in shared memory, one (key, count, min year) record per
 * block -- into the partition of the top bits of its key's hash; one block
 * per partition then aggregates the partition in a shared-memory table, so
 * the group table never leaves the SM however many groups there are.  The
 * caller picks the fan-out (the MLP's predicted group count: one partition
 * while the single-pass table stays in L2, else enough partitions for a few
 * thousand groups each).  The record buffers hold one record per B row (a
 * survivor makes at most one) while that stays within 16 GiB, else they are
 * sized from predicted_joined_rows.  A record buffer or partition table that
 * turns out too small sets overflowed; bo_groupby_topk_partitioned then
 * reruns the plain form. */
#define BO_GB_MAX_LOG2_PARTITIONS 14
int bo_groupby_topk_partitioned_device(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b,
                                       const bo_gb_c_cols* c, const bo_gb_params* params, int32_t log2_partitions,
                                       float predicted_joined_rows, bo_gb_result* out_device);
int bo_groupby_topk_partitioned(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b, const bo_gb_c_cols* c,
                                const bo_gb_params* params, int32_t log2_partitions, float predicted_joined_rows,
                                bo_gb_result* out_host);
/* Bitmap of A's ids over [0, a_id_max] ((a_id_max + 32) / 32 words, device),
 * the semi-join mask of the group-by (the reference rebuilds such masks per
 * query, e.g. build_id_mask in bespoke_ceb/query_q1a.cpp); it depends only on
 * A, so it can be built once when the table is loaded.  Asynchronous. */
int bo_groupby_a_mask_device(bo_ctx* ctx, const bo_gb_a_cols* a, int32_t a_id_max, uint32_t* mask_device);
/* The exact pre-pass alone: out_device[0] = distinct qualifying groups,
 * out_device[1] = joined rows (device int64[2]); asynchronous. */
int bo_groupby_distinct_device(bo_ctx* ctx, const bo_gb_a_cols* a, const bo_gb_b_cols* b, const bo_gb_c_cols* c,
                               const bo_gb_params* params, int64_t* out_device);

/* ================================================================== SORT ==
 * Stable LSD onesweep radix sort (decoupled look-back) of (uint64 key, uint32
 * value) pairs ascending by key bits [begin_bit, end_bit).  Replaces the LSD
 * counting sorts of bespoke_tpch/query_q10.cpp:134-168, 285-316, 318-372. */
int bo_radix_sort_pairs_device(bo_ctx* ctx, uint64_t* keys, uint32_t* vals, int64_t n, int32_t begin_bit,
                               int32_t end_bit);
int bo_radix_sort_pairs_host(bo_ctx* ctx, uint64_t* keys, uint32_t* vals, int64_t n, int32_t begin_bit,
                             int32_t end_bit);

/* ================================================================ TPC-H Q3 ==
 * run_q3 over the storage-plan layout (bespoke_tpch/query_q3.cpp:153-365):
 * customers of one market segment, their orders dated before D, each order's
 * revenue = sum of discounted_price over its lineitems shipped after D; every
 * order with such a lineitem, sorted by revenue desc, orderdate asc (rows equal
 * in both come in orderkey order).  Columns as the reference builder lays them
 * out (bespoke_tpch/builder_impl.hpp:39-97): dates are int16 day offsets from
 * the database's base date, orders sorted by orderdate, orderkey_to_row maps an
 * orderkey to its orders row (-1 if none; builder_impl.cpp:610-642). */
typedef struct bo_tpch_q3_tables {
  const int32_t* c_custkey;
  const uint16_t* c_mktsegment;   /* dictionary codes */
  int64_t n_customer;
  int32_t custkey_bound;          /* max custkey + 1 (0 if none) */
  int32_t pad0;
  const int32_t* o_orderkey;
  const int32_t* o_custkey;
  const int16_t* o_orderdate;
  const int32_t* o_shippriority;  /* may be NULL (reported as 0) */
  int64_t n_orders;
  const int32_t* orderkey_to_row;
  int64_t n_orderkey_map;
  const int32_t* l_orderkey;
  const int16_t* l_shipdate;
  const int32_t* l_discounted_price;
  int64_t n_lineitem;
} bo_tpch_q3_tables;

typedef struct bo_tpch_q3_row {   /* Q3ResultRow fields (bespoke_tpch/query_q3.hpp:10-15) */
  int64_t revenue_raw;            /* x100 */
  int32_t orderkey;
  int32_t shippriority;
  int16_t orderdate_offset;
  int16_t pad0;
  int32_t pad1;
} bo_tpch_q3_row;

/* Device columns in, rows on the host: the first min(n, max_rows) rows are
 * written to out_host and *n_rows = n.  segment_code < 0 (segment not in the
 * dictionary) gives no rows.  Where out_host is mapped pinned host memory
 * (bo_host_alloc_pinned; 16-byte aligned) the last kernel writes the rows
 * into it directly and the call synchronises once; other memory receives a
 * copy.  The same holds for bo_tpch_q11_rows, bo_tpch_q16 and bo_tpch_q2. */
int bo_tpch_q3(bo_ctx* ctx, const bo_tpch_q3_tables* tables, int16_t date_offset, int32_t segment_code,
               bo_tpch_q3_row* out_host, int64_t max_rows, int64_t* n_rows);

/* ===================================================== TPC-H order ranges ==
 * Build step of the reference's per-order lineitem ranges
 * (bespoke_tpch/builder_impl.cpp:930-990): for each orders row r,
 * [begin[r], end[r]) spans the first to the last lineitem whose orderkey maps
 * to r through orderkey_to_row; end[r] == 0 when none does.  For lineitems
 * sorted by orderkey that is the orderkey's run, as in the reference's sorted
 * branch; otherwise the same min / max bounds as its unsorted branch.  Device
 * pointers; n_lineitem < 2^32. */
int bo_tpch_order_ranges(bo_ctx* ctx, const int32_t* l_orderkey, int64_t n_lineitem, const int32_t* orderkey_to_row,
                         int64_t n_orderkey_map, int64_t n_orders, uint32_t* begin, uint32_t* end);

/* =============================================================== TPC-H Q10 ==
 * run_q10 over the storage-plan layout (bespoke_tpch/query_q10.cpp:375-585):
 * orders dated in [start, end) (orders sorted by orderdate, so these are the
 * reference's lower_bound range, :411-424) whose custkey is in
 * [0, n_custkey_map); each order's revenue = sum of discounted_price over the
 * lineitems of its range with a group code in [group_lo, group_lo +
 * group_count) (returnflag 'R' x every linestatus, :396-405), checking the
 * lineitem's orderkey unless lineitem_orderkey_sorted (:450-476); orders with
 * revenue != 0 add it to their customer; every such customer that has a row
 * (custkey_to_row >= 0) and a nationkey in [0, nation_bound), sorted by
 * revenue descending as an unsigned 64-bit value (:352-371), then custkey
 * ascending. */
typedef struct bo_tpch_q10_tables {
  const int32_t* o_orderkey;
  const int32_t* o_custkey;
  const int16_t* o_orderdate;         /* ascending */
  const uint32_t* o_li_begin;         /* bo_tpch_order_ranges */
  const uint32_t* o_li_end;
  int64_t n_orders;
  const int32_t* l_orderkey;
  const uint8_t* l_returnflag_linestatus;
  const int32_t* l_discounted_price;  /* x100 */
  int64_t n_lineitem;
  int32_t lineitem_orderkey_sorted;   /* l_orderkey non-decreasing (builder_impl.cpp:569-577) */
  int32_t nation_bound;               /* max(0, max n_nationkey) + 1 */
  const int32_t* custkey_to_row;      /* last customer row of each custkey >= 0; -1 if none */
  int64_t n_custkey_map;              /* max custkey + 1 (0 if no customer) */
  const int32_t* c_nationkey;         /* per customer row */
  int64_t n_customer;
  /* Optional (all NULL: not gathered): per customer row the string offsets of
   * the host's name / address / phone / comment columns (n_customer + 1
   * each: row i's bytes are [off[i], off[i + 1])) and acctbal (x100).  Given,
   * each result row carries its customer's ranges and balance, so the host
   * materialises Q10ResultRow without random reads of its own. */
  const uint32_t* c_name_offsets;
  const uint32_t* c_address_offsets;
  const uint32_t* c_phone_offsets;
  const uint32_t* c_comment_offsets;
  const int32_t* c_acctbal;
} bo_tpch_q10_tables;

typedef struct bo_tpch_q10_row {      /* Q10ResultRow keys (bespoke_tpch/query_q10.hpp:10-19) */
  int64_t revenue_raw;                /* x100 */
  int32_t custkey;
  int32_t cust_row;                   /* customer row: name, acctbal, address, phone, comment */
  int32_t nationkey;
  int32_t acctbal_raw;                /* x100; 0 unless the tables carry c_acctbal */
  /* [begin, begin + len) of the customer's strings in the host columns
   * (0, 0 unless the tables carry the offsets) */
  uint32_t name_begin, name_len, address_begin, address_len;
  uint32_t phone_begin, phone_len, comment_begin, comment_len;
} bo_tpch_q10_row;

/* Device columns in, rows on the host (first min(n, max_rows); *n_rows = n).
 * group_lo < 0 ('R' not in the returnflag dictionary) gives no rows. */
int bo_tpch_q10(bo_ctx* ctx, const bo_tpch_q10_tables* tables, int16_t start_offset, int16_t end_offset,
                int32_t group_lo, int32_t group_count, bo_tpch_q10_row* out_host, int64_t max_rows,
                int64_t* n_rows);

/* A host string: bytes [ptr, ptr + len) in host memory. */
typedef struct bo_host_str {
  const char* ptr;
  uint64_t len;
} bo_host_str;

/* The host's copies of the strings a Q10 result row shows: the customer
 * columns' bytes (the offset columns of the tables index them) and the name
 * of each nation key 0 .. n_nation - 1 (n_nation >= the tables' nation_bound). */
typedef struct bo_tpch_q10_host_strings {
  const char* name_data;
  const char* address_data;
  const char* phone_data;
  const char* comment_data;
  const bo_host_str* nation_names;     /* host array */
  int32_t n_nation;
  int32_t pad;
} bo_tpch_q10_host_strings;

/* Q10ResultRow (bespoke_tpch/query_q10.hpp:10-19) with its strings as host
 * pointers. */
typedef struct bo_tpch_q10_host_row {
  int32_t custkey;
  int32_t acctbal_raw;                 /* x100 */
  int64_t revenue_raw;                 /* x100 */
  bo_host_str name, nation_name, address, phone, comment;
} bo_tpch_q10_host_row;

/* bo_tpch_q10 with the rows finished on the device: the last kernel writes
 * each row, its strings resolved to host pointers, straight into rows_mapped,
 * which must be mapped pinned host memory (bo_host_alloc_pinned); no copy
 * and no host pass follow, so the rows are complete when the call returns.
 * The tables must carry the four offset columns and c_acctbal. */
int bo_tpch_q10_host_rows(bo_ctx* ctx, const bo_tpch_q10_tables* tables, int16_t start_offset, int16_t end_offset,
                          int32_t group_lo, int32_t group_count, const bo_tpch_q10_host_strings* strings,
                          bo_tpch_q10_host_row* rows_mapped, int64_t max_rows, int64_t* n_rows);

/* =============================================================== TPC-H Q18 ==
 * run_q18 over the storage-plan layout (bespoke_tpch/query_q18.cpp:183-455):
 * sum_qty[k] = sum of l_quantity over the lineitems of orderkey k; orders
 * whose sum exceeds the threshold, with their customer, sorted by totalprice
 * desc, orderdate asc, orderkey asc.  The reference's two paths:
 *   dense_orderkeys (the date-sorted orders start with orderkey 1 and end with
 *   orderkey n_orders, :204-206): lineitem orderkeys index [0, n_orders]
 *   (others are an error here); orderkey k in [1, n_orders] qualifies and
 *   reads orders row k - 1 (:207-290); its customer row is custkey - 1 when
 *   dense_custkeys, else custkey_to_row;
 *   otherwise: sums over [0, orderkey_bound); every orders row whose
 *   orderkey's sum exceeds the threshold, customer row from custkey_to_row
 *   (:292-434).
 * The dense path qualifies an order when its running sum first exceeds the
 * threshold (:232-238); with negative quantities that differs from the final
 * sum, so a negative quantity there is an error.  A custkey outside the map
 * has no customer row (the reference reads past its map there). */
typedef struct bo_tpch_q18_tables {
  const int32_t* o_orderkey;          /* date-sorted orders */
  const int32_t* o_custkey;
  const int16_t* o_orderdate;
  const int32_t* o_totalprice;        /* x100 */
  int64_t n_orders;
  const int32_t* l_orderkey;          /* 16-byte aligned */
  const int16_t* l_quantity;          /* x100, 16-byte aligned */
  int64_t n_lineitem;
  const int32_t* custkey_to_row;      /* last customer row of each custkey >= 0; -1 if none */
  int64_t n_custkey_map;              /* max custkey + 1 (0 if no customer) */
  int64_t n_customer;
  int64_t orderkey_bound;             /* max(max o_orderkey, max l_orderkey) + 1 */
  int32_t dense_orderkeys;
  int32_t dense_custkeys;             /* customer keys start at 1 and end at n_customer */
} bo_tpch_q18_tables;

typedef struct bo_tpch_q18_row {      /* Q18ResultRow fields (bespoke_tpch/query_q18.hpp:10-17) */
  int64_t sum_qty_raw;                /* x100 */
  int32_t custkey;
  int32_t cust_row;                   /* customer row: c_name */
  int32_t orderkey;
  int32_t totalprice_raw;             /* x100 */
  int16_t orderdate_offset;
  int16_t pad0;
  int32_t pad1;
} bo_tpch_q18_row;

/* quantity_threshold x100 (llround of QUANTITY * 100, :198-199).  Rows as in
 * bo_tpch_q10. */
int bo_tpch_q18(bo_ctx* ctx, const bo_tpch_q18_tables* tables, int32_t quantity_threshold,
                bo_tpch_q18_row* out_host, int64_t max_rows, int64_t* n_rows);

/* =============================================================== TPC-H Q13 ==
 * run_q13 (bespoke_tpch/query_q13.cpp:166-270): per custkey, the orders whose
 * comment does NOT match word1 ... word2; then, per customer row, how many
 * customers have each order count (c_count -> custdist), sorted by custdist
 * desc, c_count desc.  The match is the reference's (:44-83): word1's first
 * occurrence p, then word2 at or after p + len1; an empty word matches at the
 * search start, but a search that starts at the comment's end finds nothing.
 * (The reference's alpha / bigram masks only skip rows that cannot match.)
 * An order whose custkey is outside [0, n_count_map) is an error (the
 * reference indexes past its array there). */
typedef struct bo_tpch_q13_tables {
  const uint8_t* o_comment;           /* concatenated comment bytes, 16-byte aligned */
  const uint32_t* o_comment_offsets;  /* n_orders + 1; comment i is [off[i], off[i + 1]) */
  const int32_t* o_custkey;
  int64_t n_orders;
  const int32_t* c_custkey;
  int64_t n_customer;
  int64_t n_count_map;                /* max custkey + 1 */
} bo_tpch_q13_tables;

typedef struct bo_tpch_q13_row {      /* Q13ResultRow (bespoke_tpch/query_q13.hpp:9-12) */
  int64_t c_count;
  int64_t custdist;
} bo_tpch_q13_row;

/* word1 / word2: host bytes (not NUL-terminated).  Rows as in bo_tpch_q10. */
int bo_tpch_q13(bo_ctx* ctx, const bo_tpch_q13_tables* tables, const char* word1, int64_t len1, const char* word2,
                int64_t len2, bo_tpch_q13_row* out_host, int64_t max_rows, int64_t* n_rows);

/* TPC-H Q5 over the storage-plan layout: run_q5 of
 * bespoke_tpch/query_q5.cpp:197-540.  Orders dated in [start_offset,
 * end_offset) whose customer's nation (o_cust_nation, the builder's
 * orders.cust_nationkey, builder_impl.cpp:913-928) is in the region
 * (nation_in_region_host[nation] != 0, n_nations entries), summing the
 * discounted price of the lineitems in their range whose supplier's nation
 * (l_supp_nation, builder_impl.cpp:838-853) is that same nation; with
 * lineitems not sorted by orderkey only the range's lineitems of the order's
 * own key count.  revenue_out holds n_nations int64 sums. */
typedef struct bo_tpch_q5_tables {
  const int32_t* o_orderkey;
  const int16_t* o_orderdate;          /* sorted ascending */
  const int16_t* o_cust_nation;        /* -1: no customer row */
  const uint32_t* o_li_begin;
  const uint32_t* o_li_end;
  int64_t n_orders;
  const int32_t* l_orderkey;
  const int16_t* l_supp_nation;        /* -1: no supplier row */
  const int32_t* l_discounted_price;
  int64_t n_lineitem;
  int32_t lineitem_orderkey_sorted;
  int32_t n_nations;                   /* max nationkey + 1 */
} bo_tpch_q5_tables;

int bo_tpch_q5(bo_ctx* ctx, const bo_tpch_q5_tables* tables, const uint8_t* nation_in_region_host,
               int16_t start_offset, int16_t end_offset, int64_t* revenue_out);

/* TPC-H Q4 over the storage-plan layout: run_q4 of
 * bespoke_tpch/query_q4.cpp:172-355.  Orders dated in [start_offset,
 * end_offset) (the date-sorted rows the reference finds by lower_bound,
 * :190-197) with at least one lineitem in their range whose commit date is
 * before its receipt date, compared as unsigned 16-bit offsets (q4_is_late,
 * :71-73), counted by order-priority code.  With lineitems not sorted by
 * orderkey only the range's lineitems of the order's own key count (:259-311).
 * counts_out holds n_priorities counts. */
typedef struct bo_tpch_q4_tables {
  const int32_t* o_orderkey;
  const int16_t* o_orderdate;          /* sorted ascending */
  const uint16_t* o_orderpriority;     /* dictionary codes < n_priorities */
  const uint32_t* o_li_begin;          /* per-order lineitem range; end 0 = none */
  const uint32_t* o_li_end;
  int64_t n_orders;
  const int32_t* l_orderkey;
  const uint32_t* l_commit_receipt;    /* (uint16)receipt << 16 | (uint16)commit */
  int64_t n_lineitem;
  int32_t lineitem_orderkey_sorted;
  int32_t n_priorities;
} bo_tpch_q4_tables;

int bo_tpch_q4(bo_ctx* ctx, const bo_tpch_q4_tables* tables, int16_t start_offset, int16_t end_offset,
               int64_t* counts_out);

/* TPC-H Q14 over the storage-plan layout: run_q14 of
 * bespoke_tpch/query_q14.cpp:176-352.  Lineitems shipped in [start_offset,
 * end_offset) whose partkey has a part row: sums_out[1] = the sum of their
 * discounted prices, sums_out[0] = the same over parts whose type starts
 * with PROMO (int64, as the reference's promo_sum / total_sum).
 * p_promo_by_key[k] = 1 (promo type), 0 (other type) or -1 (no part row
 * with key k), the reference's partkey_promo (:193-223), built once by the
 * drop-in's build(). */
typedef struct bo_tpch_q14_tables {
  const int16_t* l_shipdate;           /* 16-byte aligned */
  const int32_t* l_partkey;
  const int32_t* l_discounted_price;
  int64_t n_lineitem;
  const int8_t* p_promo_by_key;
  int64_t n_promo_map;                 /* max partkey + 1 */
} bo_tpch_q14_tables;

int bo_tpch_q14(bo_ctx* ctx, const bo_tpch_q14_tables* tables, int16_t start_offset, int16_t end_offset,
                int64_t sums_out[2]);

/* TPC-H Q7 over the storage-plan layout: run_q7 of
 * bespoke_tpch/query_q7.cpp:140-435.  Lineitems shipped in [ship_start,
 * ship_last] (both ends included) whose supplier is tagged (supp_tag_host:
 * per suppkey 0 = the first nation, 1 = the second, -1 = neither, the
 * reference's supp_tag :170-181) and whose order's customer nation
 * (o_cust_nation) is nation1 (0) or, when the nations differ, nation2 (1);
 * pairs of the same nation count only when nation1 == nation2.  The
 * discounted price is summed into revenue_out[supp * 4 + cust * 2 + year],
 * year 1 from year2_start on.  Suppkeys outside the tag table are untagged. */
typedef struct bo_tpch_q7_tables {
  const int16_t* l_shipdate;           /* 16-byte aligned */
  const int32_t* l_suppkey;
  const int32_t* l_orderkey;
  const int32_t* l_discounted_price;
  int64_t n_lineitem;
  const int32_t* orderkey_to_row;
  int64_t n_orderkey_map;
  const int16_t* o_cust_nation;
  int64_t n_orders;
} bo_tpch_q7_tables;

int bo_tpch_q7(bo_ctx* ctx, const bo_tpch_q7_tables* tables, const int8_t* supp_tag_host, int64_t n_supp_tag,
               int32_t nation1, int32_t nation2, int16_t ship_start, int16_t ship_last, int16_t year2_start,
               int64_t revenue_out[8]);

/* TPC-H Q8 over the storage-plan layout: run_q8 of
 * bespoke_tpch/query_q8.cpp:122-380.  Lineitems of parts of the given type
 * code whose order (through orderkey_to_row) is dated in [date_start,
 * date_last] and placed by a customer of a nation in the region
 * (nation_in_region_host, n_nations bytes; a custkey qualifies when any of
 * its customer rows does, :160-167): the volume extendedprice *
 * (100 - discount) summed per order year (index 1 from year2_start on) into
 * sums_out[2 + year], and into sums_out[year] when the lineitem's supplier
 * is of the target nation (supp_target_host, per suppkey, :169-176).
 * Keys outside a table match nothing. */
typedef struct bo_tpch_q8_tables {
  const int32_t* l_partkey;            /* 32-byte aligned */
  const int32_t* l_suppkey;
  const int32_t* l_orderkey;
  const int32_t* l_extendedprice;
  const uint8_t* l_discount;
  int64_t n_lineitem;
  const int32_t* orderkey_to_row;
  int64_t n_orderkey_map;
  const int32_t* o_custkey;
  const int16_t* o_orderdate;
  int64_t n_orders;
  const int32_t* c_custkey;
  const int32_t* c_nationkey;
  int64_t n_customer;
  int32_t max_custkey;                 /* < 0: no customers */
  int32_t max_partkey;                 /* < 0: no parts */
  const int32_t* p_partkey;
  const uint16_t* p_type;              /* dictionary codes */
  int64_t n_part;
} bo_tpch_q8_tables;

int bo_tpch_q8(bo_ctx* ctx, const bo_tpch_q8_tables* tables, const uint8_t* nation_in_region_host, int32_t n_nations,
               const uint8_t* supp_target_host, int64_t n_supp, int32_t type_code, int16_t date_start,
               int16_t date_last, int16_t year2_start, int64_t sums_out[4]);

/* TPC-H Q22 over the storage-plan layout: run_q22 of
 * bespoke_tpch/query_q22.cpp:272-540.  A customer's phone class is its
 * numeric two-digit prefix (c_phone_prefix, 0..99; 255 otherwise) or, when
 * that is 255, one of the n_extra non-numeric two-character prefixes
 * (extra_pairs: (c0 << 8) | c1; c_phone_pair = 0x10000 | (c0 << 8) | c1 for
 * phones of two characters or more, else 0).  Over the customers of an
 * allowed class with a positive balance, avg = sum / count (int64); then the
 * customers of an allowed class with a balance above avg whose custkey has
 * no order (o_has_order bit clear; custkeys beyond n_order_custkeys count as
 * without orders) are counted per class: counts_out / sums_out[code] for
 * numeric classes 0..99, [100 + i] for extra prefix i (n_extra <= 7). */
typedef struct bo_tpch_q22_tables {
  const int32_t* c_custkey;
  const int32_t* c_acctbal;            /* x100 */
  const uint8_t* c_phone_prefix;
  const uint32_t* c_phone_pair;
  int64_t n_customer;
  const uint32_t* o_has_order;         /* bit per custkey */
  int64_t n_order_custkeys;
} bo_tpch_q22_tables;

#define BO_Q22_MAX_EXTRA 7
int bo_tpch_q22(bo_ctx* ctx, const bo_tpch_q22_tables* tables, const uint8_t numeric_allowed[100],
                const uint16_t* extra_pairs, int32_t n_extra, int64_t counts_out[107], int64_t sums_out[107]);

/* TPC-H Q11 over the storage-plan layout: run_q11 of
 * bespoke_tpch/query_q11.cpp:109-224.  Over the partsupp rows whose
 * supplier is in the nation (supp_in_nation_host, per suppkey, n_supp
 * bytes; suppkeys outside it are not), the value supplycost * availqty
 * (x100, the builder's supplycost_availqty) summed into
 * sums_out[partkey - min_partkey] (max_partkey - min_partkey + 1 entries)
 * and into *total_out.  Every partsupp partkey lies in [min, max]. */
typedef struct bo_tpch_q11_tables {
  const int32_t* ps_partkey;
  const int32_t* ps_suppkey;
  const int32_t* ps_value;
  int64_t n_partsupp;
  int32_t min_partkey;
  int32_t max_partkey;
} bo_tpch_q11_tables;

int bo_tpch_q11(bo_ctx* ctx, const bo_tpch_q11_tables* tables, const uint8_t* supp_in_nation_host, int64_t n_supp,
                int64_t* sums_out, int64_t* total_out);

/* Q11's result rows on the device (query_q11.cpp:186-210): partkeys whose
 * non-zero sum exceeds (double)total * fraction, by value descending then
 * partkey.  *n_rows counts them; rows past max_rows are not written. */
typedef struct bo_tpch_q11_row {
  int32_t ps_partkey;
  int32_t pad;
  int64_t value_raw;
} bo_tpch_q11_row;

int bo_tpch_q11_rows(bo_ctx* ctx, const bo_tpch_q11_tables* tables, const uint8_t* supp_in_nation_host,
                     int64_t n_supp, double fraction, bo_tpch_q11_row* rows_out, int64_t max_rows, int64_t* n_rows);

/* TPC-H Q15 over the storage-plan layout: run_q15 of
 * bespoke_tpch/query_q15.cpp:215-534.  The discounted prices of lineitems
 * shipped in [start_offset, end_offset), summed per suppkey into
 * revenue_out[0 .. n_supp) (suppkeys outside it are not summed);
 * *shipped_out = the number of lineitems in the window (the reference
 * returns no rows when it is 0, :454-456). */
typedef struct bo_tpch_q15_tables {
  const int16_t* l_shipdate;           /* 16-byte aligned */
  const int32_t* l_suppkey;
  const int32_t* l_discounted_price;
  int64_t n_lineitem;
} bo_tpch_q15_tables;

int bo_tpch_q15(bo_ctx* ctx, const bo_tpch_q15_tables* tables, int64_t n_supp, int16_t start_offset,
                int16_t end_offset, int64_t* revenue_out, int64_t* shipped_out);

/* TPC-H Q17 over the storage-plan layout: run_q17 of
 * bespoke_tpch/query_q17.cpp:119-311.  Parts with keys in [0, max_partkey]
 * of the given brand and container codes; the lineitems of those parts,
 * their quantity sum and count per part; *sum_out = the sum of the
 * extended prices of those lineitems with 5 * quantity * count < sum (the
 * reference's integer form of quantity < 0.2 * avg).  Lineitem partkeys are
 * read as unsigned and beyond max_partkey match no part. */
typedef struct bo_tpch_q17_tables {
  const int32_t* l_partkey;            /* 32-byte aligned */
  const int16_t* l_quantity;
  const int32_t* l_extendedprice;
  int64_t n_lineitem;
  const int32_t* p_partkey;
  const uint16_t* p_brand;             /* dictionary codes */
  const uint16_t* p_container;
  int64_t n_part;
  int32_t max_partkey;                 /* largest part key; < 0: none */
  int32_t pad;
} bo_tpch_q17_tables;

int bo_tpch_q17(bo_ctx* ctx, const bo_tpch_q17_tables* tables, int32_t brand_code, int32_t container_code,
                int64_t* sum_out);

/* TPC-H Q9 over the storage-plan layout: run_q9 of
 * bespoke_tpch/query_q9.cpp:130-447.  Parts whose name contains `color`
 * (byte substring, :147-150; an empty color matches every name) with keys in
 * [0, n_part_keys); their lineitems whose (partkey, suppkey) has a partsupp
 * row -- the first of the partkey's rows in partsupp order with that
 * suppkey (:160-186 and the slot scans of :262-300) -- add
 * discounted_price - supplycost * quantity / 100 (int64, truncated) to
 * totals_out[supp_nation * year_span + year], year = o_year_by_key[orderkey]
 * (the order's year minus the first order year; 255 = no order), and set
 * used_out at the same index (:313-318).  partsupp is sorted by partkey
 * (stable, as the builder sorts it); ps_part_begin[k] .. ps_part_begin[k+1]
 * are partkey k's rows (n_part_keys + 1 offsets).  slots_per_part is the
 * largest row count of a partkey: when it is 4 the reference tests all four
 * slots of every part, and the empty ones carry suppkey -1 and cost 0
 * (:262-291), which this entry point reproduces.  Lineitems with a negative
 * supplier nation, a nation at or beyond nation_bound, an orderkey outside
 * o_year_by_key or a year offset at or beyond year_span, or a partkey outside
 * [0, n_part_keys) add nothing (the reference reads out of bounds there). */
typedef struct bo_tpch_q9_tables {
  const int32_t* l_partkey;            /* 32-byte aligned */
  const int32_t* l_suppkey;
  const int32_t* l_orderkey;
  const int16_t* l_quantity;           /* x100 */
  const int32_t* l_discounted_price;   /* x100 */
  const int16_t* l_supp_nation;
  int64_t n_lineitem;
  const char* p_name;                  /* part names, concatenated */
  const uint32_t* p_name_offsets;      /* n_part + 1 */
  const int32_t* p_partkey;
  int64_t n_part;
  const int32_t* ps_suppkey;           /* partsupp sorted by partkey */
  const int32_t* ps_supplycost;        /* x100 */
  const int32_t* ps_part_begin;        /* n_part_keys + 1 */
  int64_t n_part_keys;                 /* largest part / partsupp key + 1 */
  int32_t slots_per_part;
  int32_t pad;
  const uint8_t* o_year_by_key;
  int64_t n_orderkeys;
} bo_tpch_q9_tables;

int bo_tpch_q9(bo_ctx* ctx, const bo_tpch_q9_tables* tables, const char* color, int32_t color_len,
               int32_t nation_bound, int32_t year_span, int64_t* totals_out, uint8_t* used_out);

/* The order-year table run_q9 derives (bespoke_tpch/query_q9.cpp:188-226):
 * out_device[k] = year(orderdate of row orderkey_to_row[k]) - first_year
 * (the map keeps the last date-sorted row of each orderkey, as run_q9's loop
 * over the rows does), 255 where the map holds no row; n_keys entries.
 * year_by_date_host holds the year of each date offset in
 * [min_orderdate, min_orderdate + n_dates). */
int bo_tpch_order_years(bo_ctx* ctx, const int32_t* orderkey_to_row, int64_t n_keys, const int16_t* o_orderdate,
                        int64_t n_orders, int16_t min_orderdate, const int16_t* year_by_date_host, int32_t n_dates,
                        int32_t first_year, uint8_t* out_device);

/* TPC-H Q19 over the storage-plan layout: run_q19 of
 * bespoke_tpch/query_q19.cpp:130-338.  A partkey k in [0, n_mask) belongs to
 * group g (bit g of its mask, g = 0, 1, 2) when the last part row of k
 * (p_row_by_key[k]; -1 = no part row, mask 0) has brand_code[g] (-1: group
 * off or brand unknown), a container whose code has bit g set in
 * container_groups_host[code] (n_containers bytes) and a size in
 * [1, size_high[g]].  Lineitems with shipmode code mode1 or mode2 (-1:
 * none), shipinstruct code instruct_code, a partkey in [0, n_mask) whose
 * mask is non-zero and a quantity (x100) in [qty_low[g], qty_low[g] + 1000]
 * for a group of the mask add extendedprice * (100 - discount) to
 * *revenue_out (x1e4).  Partkeys outside [0, n_mask) add nothing (the
 * reference reads out of bounds there). */
typedef struct bo_tpch_q19_tables {
  const uint16_t* l_shipmode;          /* dictionary codes, 16-byte aligned */
  const uint16_t* l_shipinstruct;      /* dictionary codes, 16-byte aligned */
  const int32_t* l_partkey;
  const int16_t* l_quantity;           /* x100 */
  const int32_t* l_extendedprice;      /* x100 */
  const uint8_t* l_discount;           /* x100 */
  int64_t n_lineitem;
  const int32_t* p_row_by_key;         /* last part row of each key, -1 = none */
  int64_t n_part_keys;                 /* entries of p_row_by_key */
  const uint16_t* p_brand;             /* dictionary codes per part row */
  const uint16_t* p_container;
  const int32_t* p_size;
  int64_t n_part;
  int64_t n_mask;                      /* largest part / lineitem partkey + 1 */
} bo_tpch_q19_tables;

int bo_tpch_q19(bo_ctx* ctx, const bo_tpch_q19_tables* tables, const int32_t brand_code[3],
                const uint8_t* container_groups_host, int32_t n_containers, const int32_t size_high[3],
                const int32_t qty_low[3], int32_t mode1, int32_t mode2, int32_t instruct_code, int64_t* revenue_out);

/* TPC-H Q21 over the storage-plan layout: run_q21 of
 * bespoke_tpch/query_q21.cpp:145-392.  For every (date-sorted) order whose
 * orderstatus code is final_code and whose lineitem range holds more than one
 * row: its lineitems (in the unsorted layout only those with the order's key)
 * with a suppkey in [0, max_suppkey] are walked; the order counts when they
 * name more than one supplier and every late one (receipt > commit, both as
 * unsigned 16-bit offsets) has the same supplier, and that supplier is a
 * target (target_host, max_suppkey + 1 bytes): its wait count (waits_out,
 * max_suppkey + 1 entries) grows by the order's late lineitems.  The walk
 * stops at a second late supplier (:257-266). */
typedef struct bo_tpch_q21_tables {
  const int32_t* l_orderkey;
  const int32_t* l_suppkey;
  const uint32_t* l_commit_receipt;    /* receipt << 16 | commit */
  int64_t n_lineitem;
  const int32_t* o_orderkey;
  const uint16_t* o_orderstatus;       /* dictionary codes */
  const uint32_t* o_li_begin;
  const uint32_t* o_li_end;
  int64_t n_orders;
  int32_t lineitem_orderkey_sorted;
  int32_t pad;
} bo_tpch_q21_tables;

int bo_tpch_q21(bo_ctx* ctx, const bo_tpch_q21_tables* tables, int32_t final_code, const uint8_t* target_host,
                int32_t max_suppkey, int64_t* waits_out);

/* ==================================================================== CEB ==
 * The reference's CEB engine keeps every column as values plus a null byte
 * per row (ColumnData, bespoke_ceb/builder_impl.hpp:97-111): int32 values
 * (0 where null) and, for strings, ids into a string pool.  The GPU form is
 * the same layout per column: int32 values (string columns: codes of the
 * column's dictionary) and an optional is_null byte array (NULL: the column
 * has no nulls). */
typedef struct bo_ceb_col {
  const int32_t* values;
  const uint8_t* is_null;
} bo_ceb_col;

/* CEB query 1a: run_q1a of bespoke_ceb/query_q1a.cpp:155-655.  Titles of an
 * allowed kind with year2 <= production_year <= year1; per title movie the
 * movie_info rows of an info type in ID1 with an info value in INFO1
 * (count1), likewise ID2 / INFO2 (count2); the cast_info rows of the movies
 * with both counts, an allowed role and an allowed person (cast count);
 * *count_out = sum over the qualifying title rows of cast * count1 * count2.
 * Rows with a null in a column the reference tests are skipped as it skips
 * them.  Kind / role / person masks come from the dimension rows whose
 * dictionary code is allowed (kind_allowed etc., one byte per code) and whose
 * id lies in [0, *_mask_size); the info-type filter holds one byte per
 * info-type id in [0, info_type_size) (bit 0: ID1, bit 1: ID2) and the info
 * match one byte per movie_info.info code (bit 0: INFO1, bit 1: INFO2).
 * Movie ids beyond the largest qualifying title id are dropped, as the
 * reference drops them; max_title_id bounds every title id. */
typedef struct bo_ceb_q1a_tables {
  bo_ceb_col t_id, t_kind_id, t_year;
  int64_t n_title;
  int32_t max_title_id;                /* largest title id (< 0: none) */
  int32_t pad0;
  bo_ceb_col mi_movie_id, mi_info_type_id, mi_info;
  int64_t n_movie_info;
  bo_ceb_col ci_movie_id, ci_person_id, ci_role_id;
  int64_t n_cast_info;
  bo_ceb_col kt_id, kt_kind;
  int64_t n_kind_type;
  bo_ceb_col rt_id, rt_role;
  int64_t n_role_type;
  bo_ceb_col nm_id, nm_gender;
  int64_t n_name;
} bo_ceb_q1a_tables;

typedef struct bo_ceb_q1a_params {
  int32_t year1, year2;
  const uint8_t* info_type_filter;     /* host */
  int32_t info_type_size;
  int32_t n_info_codes;
  const uint8_t* info_match;           /* host */
  const uint8_t* kind_allowed;         /* host, per kind code */
  const uint8_t* role_allowed;         /* host, per role code */
  const uint8_t* gender_allowed;       /* host, per gender code */
  int32_t n_kind_codes, n_role_codes, n_gender_codes;
  int32_t kind_mask_size, role_mask_size, person_mask_size;
  int32_t pad;
} bo_ceb_q1a_params;

int bo_ceb_q1a(bo_ctx* ctx, const bo_ceb_q1a_tables* tables, const bo_ceb_q1a_params* params, int64_t* count_out);

/* CEB query 10a: run_q10a of bespoke_ceb/query_q10a.cpp:334-1130 -- per
 * (person name, movie info value) the MIN and MAX production year over the
 * joined rows: titles of an allowed kind (ids in [0, n_title + 1); the last
 * row of an id gives its year, or no year when null); their movie_info rows
 * with an info type allowed by info_type_mask (one byte per id in
 * [0, info_type_size)) and an info code with a dense index in info_dense
 * (-1: not in the IN list); their cast_info rows of an allowed role with a
 * person id in [0, n_name + 1); the persons whose name (a code of the name
 * dictionary, name_dict bytes with n_name_codes + 1 offsets on the device)
 * matches the ILIKE pattern (pattern_type: 0 all, 1 exact, 2 prefix,
 * 3 suffix, 4 contains, 5 general with '%' / '_'; the token or pattern
 * lower-cased, host memory).  Groups are aggregated in a dense name-code x
 * info matrix when it has at most BO_CEB_AGG_MAX_SLOTS slots, else in a hash
 * table (the reference's switch, :843-856).  Rows (any order, as the
 * reference's) go to rows_out (host, max_rows); *n_rows_out receives the
 * group count; BO_ERR_OVERFLOW when it exceeds max_rows (nothing written).
 * *dense_out (optional) tells which aggregation ran (1 = matrix). */
#define BO_CEB_AGG_MAX_SLOTS 5000000
typedef struct bo_ceb_q10a_tables {
  bo_ceb_col t_id, t_kind_id, t_year;
  int64_t n_title;
  bo_ceb_col mi_movie_id, mi_info_type_id, mi_info;
  int64_t n_movie_info;
  bo_ceb_col ci_movie_id, ci_person_id, ci_role_id;
  int64_t n_cast_info;
  bo_ceb_col kt_id, kt_kind;
  int64_t n_kind_type;
  bo_ceb_col rt_id, rt_role;
  int64_t n_role_type;
  bo_ceb_col nm_id, nm_name;
  int64_t n_name;
  const char* name_dict;               /* device */
  const uint32_t* name_dict_offsets;   /* device, n_name_codes + 1 */
  int64_t n_name_codes;
} bo_ceb_q10a_tables;

typedef struct bo_ceb_q10a_params {
  const uint8_t* info_type_mask;       /* host */
  int32_t info_type_size;
  int32_t n_info_codes;
  const int32_t* info_dense;           /* host, per movie_info.info code */
  int32_t n_info_dense;
  int32_t n_kind_codes;
  const uint8_t* kind_allowed;         /* host, per kind code */
  const uint8_t* role_allowed;         /* host, per role code */
  int32_t n_role_codes;
  int32_t pattern_type;
  const char* pattern;                 /* host */
  int32_t pattern_len;
  int32_t pad;
} bo_ceb_q10a_params;

typedef struct bo_ceb_q10a_row {
  int32_t name_code;
  int32_t info_dense;
  int32_t has_year;
  int32_t min_year;
  int32_t max_year;
} bo_ceb_q10a_row;

int bo_ceb_q10a(bo_ctx* ctx, const bo_ceb_q10a_tables* tables, const bo_ceb_q10a_params* params,
                bo_ceb_q10a_row* rows_out, int64_t max_rows, int64_t* n_rows_out, int32_t* dense_out);

/* CEB query 3b: run_q3b of bespoke_ceb/query_q3b.cpp:728-1420 -- COUNT(*)
 * per (title, person name, company name) over movies with companies whose
 * name matches `company` (ILIKE), keywords, a title of an allowed kind that
 * matches `title`, and cast rows of an allowed role whose person's
 * name_pcode_nf matches `pcode`; the count of a movie's (person, company)
 * is keywords x cast rows x company rows (the reference's nested
 * per-movie maps, :1330-1360), summed per group and ordered by count desc,
 * then the title, name and company strings (:1369-1385; str_rank arrays give
 * each dictionary code its string order).  Movie ids are bounded by
 * movie_bound (the largest movie_companies movie id + 1), person ids by
 * person_bound.  Dictionary codes are packed into one 64-bit group key, so
 * the three dictionaries' code widths must add up to 64 bits at most
 * (BO_ERR_UNSUPPORTED otherwise).  Rows go to rows_out (host) in the
 * reference's order; BO_ERR_OVERFLOW with *n_rows_out set when there are
 * more than max_rows. */
typedef struct bo_ceb_dict {
  const char* bytes;                   /* device */
  const uint32_t* offsets;             /* device, n + 1 */
  const int32_t* rank;                 /* device: order of each code's string */
  int64_t n;
} bo_ceb_dict;

typedef struct bo_ceb_q3b_tables {
  bo_ceb_col kt_id, kt_kind;
  int64_t n_kind_type;
  bo_ceb_col rt_id, rt_role;
  int64_t n_role_type;
  bo_ceb_col cn_id, cn_name;
  int64_t n_company_name;
  bo_ceb_col mc_movie_id, mc_company_id, mc_company_type_id;
  int64_t n_movie_companies;
  bo_ceb_col mk_movie_id, mk_keyword_id;
  int64_t n_movie_keyword;
  bo_ceb_col t_id, t_title, t_kind_id;
  int64_t n_title;
  bo_ceb_col ci_movie_id, ci_person_id, ci_role_id;
  int64_t n_cast_info;
  bo_ceb_col nm_id, nm_name, nm_pcode;
  int64_t n_name;
  bo_ceb_dict title_dict, name_dict, company_dict, pcode_dict;
  int32_t movie_bound, person_bound;
} bo_ceb_q3b_tables;

typedef struct bo_ceb_q3b_params {
  const uint8_t* kind_allowed;         /* host, per kind code */
  const uint8_t* role_allowed;         /* host, per role code */
  int32_t n_kind_codes, n_role_codes;
  int32_t kind_mask_size, role_mask_size, company_map_size;
  int32_t title_type, pcode_type, company_type;  /* ILIKE kinds as for 10a */
  const char* title_pat;               /* host, lower-cased */
  const char* pcode_pat;
  const char* company_pat;
  int32_t title_len, pcode_len, company_len, pad;
} bo_ceb_q3b_params;

typedef struct bo_ceb_q3b_row {
  int32_t title_code;
  int32_t name_code;
  int32_t company_code;
  int32_t pad;
  int64_t count;
} bo_ceb_q3b_row;

int bo_ceb_q3b(bo_ctx* ctx, const bo_ceb_q3b_tables* tables, const bo_ceb_q3b_params* params,
               bo_ceb_q3b_row* rows_out, int64_t max_rows, int64_t* n_rows_out);

/* The CEB builder's fact-table order (bespoke_ceb/builder_impl.cpp:255-360,
 * 432-452): rows sorted by a primary int32 column and, optionally, a
 * secondary one (movie_info by (movie_id, info_type_id), cast_info by
 * (movie_id, role_id), movie_companies by movie_id, ...), comparing the
 * stored values (0 where null).  perm_device (n entries) receives the source
 * row of every output row; ties keep their input order (the reference's
 * std::sort leaves their order unspecified).  bo_ceb_gather_i32 / _u8 then
 * reorder a column: dst[i] = src[perm[i]]. */
int bo_ceb_sort_rows(bo_ctx* ctx, const int32_t* primary, const int32_t* secondary, int64_t n,
                     uint32_t* perm_device);
int bo_ceb_gather_i32(bo_ctx* ctx, const int32_t* src, const uint32_t* perm, int64_t n, int32_t* dst);
int bo_ceb_gather_u8(bo_ctx* ctx, const uint8_t* src, const uint32_t* perm, int64_t n, uint8_t* dst);

/* TPC-H Q12 over the storage-plan layout: run_q12 of
 * bespoke_tpch/query_q12.cpp:162-360.  Lineitems whose shipmode code is
 * mode_code1 or mode_code2 (-1: none), with shipdate < commitdate <
 * receiptdate and receiptdate in [start_offset, end_offset), joined to their
 * order through orderkey_to_row and counted by shipmode as high (order
 * priority code high_code1 or high_code2) or low.  l_shard_max_shipdate, when
 * given, is the latest shipdate of each lineitem's builder shard
 * (builder_impl.cpp:855-911); a lineitem whose shard ends more than 30 days
 * before start_offset is skipped, as the reference's sharded scan skips the
 * whole shard (:265-270).  NULL when no lineitem is received more than 30
 * days after shipping, where that pruning removes nothing.
 * counts_out[0..1] = high / low of mode_code1, [2..3] of mode_code2. */
typedef struct bo_tpch_q12_tables {
  const uint16_t* l_shipmode;          /* dictionary codes */
  const uint32_t* l_commit_receipt;    /* (uint16)receipt << 16 | (uint16)commit, int16 day offsets */
  const int16_t* l_shipdate;
  const int32_t* l_orderkey;
  const int16_t* l_shard_max_shipdate; /* optional (NULL) */
  int64_t n_lineitem;
  const int32_t* orderkey_to_row;
  int64_t n_orderkey_map;
  const uint16_t* o_orderpriority;     /* dictionary codes, orders row order */
  int64_t n_orders;
} bo_tpch_q12_tables;

int bo_tpch_q12(bo_ctx* ctx, const bo_tpch_q12_tables* tables, int32_t mode_code1, int32_t mode_code2,
                int32_t high_code1, int32_t high_code2, int16_t start_offset, int16_t end_offset,
                int64_t counts_out[4]);

/* Supplier complaint flags, the supplier scan of run_q16
 * (bespoke_tpch/query_q16.cpp:357-368, the search of :58-67): for each
 * supplier row whose comment (bytes [offsets[r], offsets[r + 1]) of
 * comments) holds "Customer" and, after it, "Complaints",
 * banned_out[suppkeys[r]] = 1.  banned_out (device, n_banned bytes) is
 * cleared first; suppkeys outside [0, n_banned) set nothing.  The flags do not
 * depend on a query's parameters, so a database computes them once. */
int bo_tpch_supplier_complaints(bo_ctx* ctx, const char* comments_device, const uint32_t* offsets_device,
                                const int32_t* suppkeys_device, int64_t n_supplier, uint8_t* banned_out,
                                int64_t n_banned);

/* TPC-H Q16 over the storage-plan layout: run_q16 of
 * bespoke_tpch/query_q16.cpp:167-541.  A part row qualifies when its brand
 * code is not banned_brand, its size s (0 <= s <= 50) has bit s of size_mask
 * set and its type code's type_banned byte is 0; a partkey k in
 * [0, n_part] takes the group (brand, type, size) of its LAST qualifying
 * row (:276-342).  A partsupp row's partkey is ps_partkey[r], or
 * r / rows_per_part + 1 when rows_per_part > 0 (the reference's walk by row
 * position when the partsupp rows are a multiple of the part rows,
 * :391-414); rows whose partkey has a group and whose suppkey is not flagged
 * in s_banned count that suppkey once per group (distinct, :449-476).  Rows
 * out: one per group with a count, by count descending, then brand, type
 * (by their ranks in string order) and size ascending (:489-521).
 * rows_out holds max_rows rows; *n_rows is the number of groups (rows past
 * max_rows are not written).  Groups: n_brand * n_type * 64 <= 2^28. */
typedef struct bo_tpch_q16_tables {
  const int32_t* p_partkey;
  const uint16_t* p_brand;             /* dictionary codes */
  const uint16_t* p_type;              /* dictionary codes */
  const int32_t* p_size;
  int64_t n_part;
  const int32_t* ps_partkey;           /* partsupp rows (stably) sorted by partkey */
  const int32_t* ps_suppkey;
  int64_t n_partsupp;
  const uint8_t* s_banned;             /* by suppkey (bo_tpch_supplier_complaints) */
  int64_t n_banned;
} bo_tpch_q16_tables;

typedef struct bo_tpch_q16_params {
  uint64_t size_mask;                  /* bit s: size s qualifies (s <= 50) */
  int32_t banned_brand;                /* brand code; -1: none */
  int32_t rows_per_part;               /* > 0: partkey of partsupp row r is r / rows_per_part + 1 */
  int32_t n_brand;                     /* brand dictionary entries */
  int32_t n_type;                      /* type dictionary entries */
  const uint16_t* brand_rank;          /* host, n_brand: rank of each code in string order */
  const uint16_t* type_rank;           /* host, n_type */
  const uint8_t* type_banned;          /* host, n_type: 1 = the type starts with the query's TYPE */
} bo_tpch_q16_params;

typedef struct bo_tpch_q16_row {
  int32_t brand_code;
  int32_t type_code;
  int32_t size;
  int32_t pad;
  int64_t supplier_cnt;
} bo_tpch_q16_row;

int bo_tpch_q16(bo_ctx* ctx, const bo_tpch_q16_tables* tables, const bo_tpch_q16_params* params,
                bo_tpch_q16_row* rows_out, int64_t max_rows, int64_t* n_rows);

/* TPC-H Q20 over the storage-plan layout: run_q20 of
 * bespoke_tpch/query_q20.cpp:338-676.  Partkeys in [0, max_partkey] whose
 * part name starts with `color` (:375-392); the quantities of lineitems
 * shipped in [start_offset, end_offset) (as (uint32)(ship - start) <
 * (uint32)(end - start), :412-421) by a supplier of nation_key with such a
 * partkey, summed per (partkey, suppkey) (:405-560 -- the builder's month
 * shards select the same rows); a partsupp row with such a partkey, a
 * supplier of nation_key and a sum with 2 * 100 * availqty > sum qualifies
 * its suppkey (:568-615).  Rows out: the supplier rows of nation_key whose
 * suppkey qualified, in s_name order (s_row_by_name: the supplier rows
 * sorted by name), :618-644.  A lineitem's (partkey, suppkey) is summed into
 * its first partsupp row of that pair (ps_part_begin: each partkey's rows);
 * pairs without a partsupp row are never looked up, as in the reference. */
typedef struct bo_tpch_q20_tables {
  const int32_t* p_partkey;
  const char* p_name;
  const uint32_t* p_name_offsets;      /* n_part + 1 */
  int64_t n_part;
  int32_t max_partkey;                 /* largest part key; < 0: none */
  int32_t max_suppkey;                 /* largest supplier key; < 0: none */
  const int16_t* l_shipdate;
  const int32_t* l_partkey;
  const int32_t* l_suppkey;
  const int16_t* l_supp_nation;        /* -1: no supplier row */
  const int16_t* l_quantity;           /* x100 */
  int64_t n_lineitem;
  const int32_t* ps_partkey;           /* partsupp rows sorted by partkey */
  const int32_t* ps_suppkey;
  const int32_t* ps_availqty;
  int64_t n_partsupp;
  const int32_t* ps_part_begin;        /* n_ps_part_keys + 1 row offsets */
  int64_t n_ps_part_keys;
  const int16_t* s_nation_by_key;      /* max_suppkey + 1 entries; -1: none */
  const int32_t* s_suppkey;
  const int32_t* s_nationkey;
  const int32_t* s_row_by_name;        /* n_supplier */
  int64_t n_supplier;
} bo_tpch_q20_tables;

int bo_tpch_q20(bo_ctx* ctx, const bo_tpch_q20_tables* tables, const char* color, int32_t color_len,
                int32_t nation_key, int16_t start_offset, int16_t end_offset, int32_t* supplier_rows_out,
                int64_t max_rows, int64_t* n_rows);

/* TPC-H Q2 over the storage-plan layout: run_q2 of
 * bespoke_tpch/query_q2.cpp:146-430.  Part rows p with size target_size and
 * a type code whose type_ok byte is set (:214-265) take partkey p + 1 (the
 * reference's assumption) and its partsupp rows (ps_part_begin); a row's
 * supplier is row suppkey - 1 (again the reference's) when below n_supplier
 * and its s_nation_idx has a set nation_ok byte (:186-212).  Of those rows,
 * the ones with the least supplycost (below INT32_MAX) each give a result
 * row (:300-381).  Rows out by s_rank[supplier row] (the row's position in
 * (acctbal desc, nation name, s_name, row) order, unique) then partkey
 * (:386-401).
 * *n_rows counts all rows; rows past max_rows are not written. */
typedef struct bo_tpch_q2_tables {
  const int32_t* p_size;
  const uint16_t* p_type;              /* dictionary codes */
  const uint16_t* p_mfgr;              /* dictionary codes */
  int64_t n_part;
  const int32_t* ps_suppkey;           /* partsupp rows sorted by partkey */
  const int32_t* ps_supplycost;        /* x100 */
  int64_t n_partsupp;
  const int32_t* ps_part_begin;        /* n_ps_part_keys + 1 row offsets */
  int64_t n_ps_part_keys;
  const int32_t* s_nation_idx;         /* nation key when below the nation row count, else -1 */
  const uint32_t* s_rank;               /* a permutation of 0 .. n_supplier - 1 */
  int64_t n_supplier;
} bo_tpch_q2_tables;

typedef struct bo_tpch_q2_row {
  int32_t partkey;
  int32_t supplier_row;
  int32_t mfgr_code;
  int32_t pad;
} bo_tpch_q2_row;

int bo_tpch_q2(bo_ctx* ctx, const bo_tpch_q2_tables* tables, int32_t target_size, const uint8_t* type_ok_host,
               int32_t n_type, const uint8_t* nation_ok_host, int32_t n_nation, bo_tpch_q2_row* rows_out,
               int64_t max_rows, int64_t* n_rows);

/* ================================================================= BATCH ==
 * Many pipelines of uneven sizes in ONE persistent kernel fed by a device work
 * queue of (instance, stage, tile) items, captured in a CUDA graph.  Stages of
 * one instance are ordered by per-instance completion counters (bounded waits);
 * work of different instances overlaps.  Tables are sized from each instance's
 * predicted count (e.g. an MLP prediction); an instance whose table overflowed
 * is rerun alone in the exact form when its results are read, so every result
 * equals the solo run.  No reference counterpart (the reference runs one query
 * at a time, bespoke_tpch/query_impl.cpp:159-388). */
#define BO_BATCH_SCAN_AGG 0
#define BO_BATCH_JOIN 1
#define BO_BATCH_GROUPBY 2
#define BO_BATCH_MAX_CATS 64

typedef struct bo_batch_instance {
  int32_t kind;            /* BO_BATCH_* */
  int32_t tile_rows;       /* largest rows per work item (tiles are smaller for small stages); 0 = default */
  float predicted;         /* join: qualifying build rows; group-by: groups; <= 0 sizes for the upper bound */
  float presize_factor;    /* slots per predicted row; 0 = the solo form's (join 4, group-by 2.5) */
  /* scan-agg (wide layout) */
  bo_fact_cols fact;
  int32_t ship_cutoff, n_flag_a, n_flag_b, pad0;
  /* join */
  bo_join_build_cols build;
  bo_join_probe_cols probe;
  bo_join_params join;
  /* group-by */
  bo_gb_a_cols a;
  bo_gb_b_cols b;
  bo_gb_c_cols c;
  uint16_t categories[BO_BATCH_MAX_CATS];
  int32_t n_categories, year_lo, year_hi, k, a_id_max, pad1;
  /* join / group-by, optional: device float read when the batch runs (e.g. an
   * MLP prediction left on the device); overrides `predicted`.  The pool then
   * holds tables of the upper-bound size and the launch uses the capacity the
   * device value gives. */
  const float* predicted_device;
} bo_batch_instance;

typedef struct bo_batch_result {
  int32_t kind;
  int32_t overflowed;   /* the batch's presized table overflowed (the result below is the exact rerun) */
  int32_t reruns;
  int32_t pad;
  bo_q1_agg q1[BO_Q1_MAX_GROUPS];
  bo_join_result join;
  bo_gb_result groupby;
} bo_batch_result;

typedef struct bo_batch bo_batch;

/* Plans a batch sized exactly for these instances: validates them, allocates
 * their tables, builds the work queue (level-major, larger instances first
 * inside a level) and captures the launch (queue reset + the persistent
 * kernel) into a CUDA graph.  workers_per_sm = 0 uses the library default. */
int bo_batch_create(bo_ctx* ctx, const bo_batch_instance* instances, int32_t n, int32_t workers_per_sm,
                    bo_batch** out);
/* An empty batch with room for max_instances instances, max_items work items
 * and pool_bytes of tables; fill it with bo_batch_update. */
int bo_batch_create_pool(bo_ctx* ctx, int32_t max_instances, int64_t max_items, int64_t pool_bytes,
                         int32_t workers_per_sm, bo_batch** out);
/* Re-plans the batch with a new set of instances inside its pool (BO_ERR_OVERFLOW
 * if their tables or items do not fit): one asynchronous copy on the
 * context's stream, no re-capture.  Read the previous launch's results first. */
int bo_batch_update(bo_ctx* ctx, bo_batch* batch, const bo_batch_instance* instances, int32_t n);
/* Table bytes and work items one instance needs (admission by footprint). */
int bo_batch_footprint(const bo_batch_instance* instance, int64_t* table_bytes, int64_t* items);
/* Launches the captured graph on the context's stream (asynchronous). */
int bo_batch_launch(bo_ctx* ctx, bo_batch* batch);
/* Waits, copies every instance's result to the host and reruns any instance
 * whose presized table overflowed alone in the exact form. */
int bo_batch_results(bo_ctx* ctx, bo_batch* batch, bo_batch_result* out_host);
/* Non-blocking: 1 if the last launch has finished, 0 if it is still running,
 * a negative status on error. */
int bo_batch_done(const bo_batch* batch);
/* Device time (ms) of the last launch, from events around the graph. */
float bo_batch_last_ms(const bo_batch* batch);
int32_t bo_batch_num_items(const bo_batch* batch);
void bo_batch_destroy(bo_batch* batch);

/* ================================================================ SKETCH ==
 * Per-column sketches for the learned sizing features, computed on the device
 * once per table.  No reference counterpart. */
#define BO_SKETCH_BINS 64
typedef struct bo_sketch {
  int64_t n;
  int64_t min, max;
  int64_t hist[BO_SKETCH_BINS];  /* equi-width over [min, max]: bin = (v-min)*64/(max-min+1) */
  double distinct_estimate;      /* HyperLogLog, 4096 registers */
} bo_sketch;
/* int32 column (device) -> sketch (host); synchronises. */
int bo_sketch_i32(bo_ctx* ctx, const int32_t* col_device, int64_t n, bo_sketch* out_host);
/* Exact histogram of a uint8 (elem_bytes 1) or uint16 (2) device column with
 * values < domain <= 65536; hist_host receives `domain` counts. */
int bo_histogram_small(bo_ctx* ctx, const void* col_device, int32_t elem_bytes, int64_t n, int32_t domain,
                       int64_t* hist_host);

/* ==================================================================== MLP ==
 * Learned sizing: a small FP32 MLP (n_features -> 64 -> 64 -> 64 -> n_outputs,
 * ReLU) trained on the GPU by its own kernels.  Targets are log1p(counts);
 * predictions presize hash tables and output buffers.  No reference
 * counterpart (the reference sizes its dense arrays exactly, e.g.
 * bespoke_tpch/query_q3.cpp:178-180).  n_features <= 32, n_outputs <= 4.
 * Parameter layout: W1[F][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64]
 * W4[64][O] b4[O] (row-major, x @ W). */
typedef struct bo_mlp bo_mlp;

int bo_mlp_create(bo_ctx* ctx, int32_t n_features, int32_t n_outputs, uint64_t seed, bo_mlp** out);
void bo_mlp_destroy(bo_mlp* mlp);
int32_t bo_mlp_num_params(const bo_mlp* mlp);
int bo_mlp_get_params(bo_ctx* ctx, const bo_mlp* mlp, float* host_out);
int bo_mlp_set_params(bo_ctx* ctx, bo_mlp* mlp, const float* host_in);
/* Gradient of the loss 0.5*mean((y - t)^2) w.r.t. every parameter (device
 * buffers: x [n][F], t [n][O], grad [P], loss [1]); deterministic. */
int bo_mlp_gradients_device(bo_ctx* ctx, bo_mlp* mlp, const float* x, const float* t, int32_t n,
                            float* grad_device, float* loss_device);
/* One Adam step on a batch (device buffers). */
int bo_mlp_train_step_device(bo_ctx* ctx, bo_mlp* mlp, const float* x, const float* t, int32_t n, float lr,
                             float* loss_device);
/* `epochs` full-batch Adam steps on host data (copied in once). */
int bo_mlp_train_host(bo_ctx* ctx, bo_mlp* mlp, const float* x_host, const float* t_host, int32_t n,
                      int32_t epochs, float lr, float* final_loss);
int bo_mlp_infer_device(bo_ctx* ctx, const bo_mlp* mlp, const float* x, int32_t n, float* y);
/* One feature vector (host, passed to the kernel by value: no copy) ->
 * counts_device[o] = max(expm1(y[o]), 0); log_device (optional) = y. */
int bo_mlp_predict_counts(bo_ctx* ctx, const bo_mlp* mlp, const float* features_host, float* counts_device,
                          float* log_device);

/* Learned join in three launches (no counterpart in the reference; the
 * presized form of the filtered join of run_q3, bespoke_tpch/query_q3.cpp:
 * 182-260): the first kernel evaluates `mlp` (output 0 = predicted qualifying
 * build rows) for the host feature vector in every block and clears the
 * table sized from it -- the result bo_mlp_predict_counts followed by
 * bo_join_presized_device gives, in one launch fewer -- then build and
 * probe.  pred_device (optional) receives the prediction.  The _device form
 * is asynchronous (out_device->overflowed reports a too-small table); the
 * host form reruns the plain form on overflow. */
int bo_join_learned_device(bo_ctx* ctx, const bo_mlp* mlp, const float* features_host,
                           const bo_join_build_cols* build, const bo_join_probe_cols* probe,
                           const bo_join_params* params, bo_join_result* out_device, float* pred_device);
int bo_join_learned(bo_ctx* ctx, const bo_mlp* mlp, const float* features_host, const bo_join_build_cols* build,
                    const bo_join_probe_cols* probe, const bo_join_params* params, bo_join_result* out_host);

#ifdef __cplusplus
}
#endif

#endif /* BESPOKE_GPU_H */
