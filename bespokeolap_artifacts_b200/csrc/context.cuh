// Host-side context shared by all entry points (internal, not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <unordered_map>
#include <vector>

#include "bespoke_gpu.h"

namespace bo {
struct GatherState;  // host threads and buffers of the streamed join's host-gather form (csrc/join.cu)
}

struct bo_ctx {
  int device = 0;
  int num_sms = 0;
  size_t l2_bytes = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string last_error;
  std::atomic<int64_t> launches{0};

  // Device error word (bo::kErr* bits) and per-operation scratch regions,
  // allocated once and kept for the context's lifetime.  Named regions are
  // grown on demand; kernels that accumulate into them leave them zeroed.
  uint32_t* d_err = nullptr;
  uint32_t* h_err = nullptr;  // pinned mirror for the single end-of-call read
  unsigned long long* h_word = nullptr;  // two pinned words: a device count (and its overflow word) read back
  struct Region {
    void* ptr = nullptr;
    size_t bytes = 0;
  };
  std::unordered_map<std::string, Region> regions;
  // Pinned staging used by the _host entry points.
  void* h_stage = nullptr;
  size_t h_stage_bytes = 0;
  // Second stream for host->device copies that overlap with kernels, and the
  // events that order the two (created on first use).
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> events;
  int stream_set = 0;  // buffer set of the streamed join's next query
  // Host threads that gather the payload of matching probe rows in the
  // streamed join (-1: chosen from the machine; 0: payload read in place).
  int gather_threads = -1;
  bo::GatherState* gather = nullptr;
};

namespace bo {

int set_error(bo_ctx* ctx, int code, const char* fmt, ...);
int cuda_fail(bo_ctx* ctx, cudaError_t e, const char* what);

#define BO_CUDA(ctx, call)                                  \
  do {                                                      \
    cudaError_t e__ = (call);                               \
    if (e__ != cudaSuccess) return bo::cuda_fail((ctx), e__, #call); \
  } while (0)

#define BO_CHECK_CTX(ctx)                                   \
  do {                                                      \
    if (!(ctx)) return BO_ERR_INVALID;                      \
  } while (0)

// Returns a device region of at least `bytes`, zero-filled when first
// allocated or grown (zeroing is ordered on the context's stream).
int region(bo_ctx* ctx, const char* name, size_t bytes, void** out);
// Pinned host staging buffer of at least `bytes`.
int host_stage(bo_ctx* ctx, size_t bytes, void** out);
// Waits for the work the context's host threads have queued (the streamed
// join's gathers) and for the device work they enqueued; reports their first
// failure.  Must not be called from those threads.
int drain_host_work(bo_ctx* ctx);
// Stops the context's host threads (after draining) and frees their buffers.
void destroy_host_work(bo_ctx* ctx);
// Records one kernel launch and checks the launch status.
int after_launch(bo_ctx* ctx, const char* what);
// Reads and clears the device error word (call only after a stream sync).
int consume_device_errors(bo_ctx* ctx, uint32_t* bits_out);
// Maps error bits to a status code with a message.
int device_error_status(bo_ctx* ctx, uint32_t bits, const char* op);
// Blocks per SM from the occupancy calculator, cached per kernel.
int occupancy_blocks(const void* kernel, int block, size_t smem);

// Next `count` elements of a workspace carved from one region, 256-byte aligned.
template <class T>
T* carve(char*& p, size_t count) {
  T* r = reinterpret_cast<T*>(p);
  p += (sizeof(T) * count + 255) & ~size_t(255);
  return r;
}

// Stable LSD radix sort of (key, value) pairs by bits [begin_bit, end_bit)
// (csrc/radix_sort.cu); n_dev, if given, is the actual count (<= n) on the
// device.  Without n_dev, up to 131,072 pairs (65,536 where the device
// schedules no 16-CTA cluster) are sorted by one thread-block cluster in
// distributed shared memory (one launch).
int radix_sort_pairs(bo_ctx* ctx, unsigned long long* keys, uint32_t* vals, unsigned long long* tmp_keys,
                     uint32_t* tmp_vals, int64_t n, int begin_bit, int end_bit, const unsigned long long* n_dev);

// The one-launch cluster sort of min(*n_dev, n_max) pairs without the count on
// the host: if the count exceeds what the largest cluster holds (kCsCap per
// CTA), *overflow is set and nothing moves (the caller then reads the count
// and sorts with radix_sort_pairs).
int cluster_sort_pairs_counted(bo_ctx* ctx, unsigned long long* keys, uint32_t* vals, const unsigned long long* n_dev,
                               int64_t n_max, int begin_bit, int end_bit, uint32_t* overflow);

// The device pointer of mapped pinned host memory (16-byte aligned), or null
// for any other pointer (pageable memory, device memory).
void* mapped_device_ptr(const void* host);

// After a pipeline whose sort read its count on the device: the count at
// n_out (clamped to n_max) and the overflow word after it (the 16 bytes at
// n_out) come back with the error word, in one synchronisation.
int read_counted(bo_ctx* ctx, const char* op, const unsigned long long* n_out, int64_t n_max, int64_t* n,
                 bool* overflow);

// Copies the device count *n_dev (clamped to n_max) to the host; synchronises
// the stream.  Lets a caller sort an exact number of pairs.
int read_device_count(bo_ctx* ctx, const unsigned long long* n_dev, int64_t n_max, int64_t* n);

// The k smallest of unique keys (ascending, k <= 64) of (keys, vals) into the
// front of (cand_keys, cand_vals): one cooperative radix-select launch
// (csrc/radix_sort.cu); tmp_keys / tmp_vals are not used.
// lo_bits / hi_max_dev (optional): keys are (hi << lo_bits) | lo with all hi
// equal above the highest bit of *hi_max_dev; the select digit sits there.
int radix_topk_pairs(bo_ctx* ctx, const unsigned long long* keys, const uint32_t* vals, int64_t n_max,
                     const unsigned long long* n_dev, int key_bits, int k, unsigned long long* cand_keys,
                     uint32_t* cand_vals, unsigned long long* tmp_keys, uint32_t* tmp_vals, int lo_bits,
                     const unsigned long long* hi_max_dev);

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
// Column pointers must be 32-byte aligned: the scans use 256-bit vector loads.
inline bool aligned32(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 31u) == 0; }

}  // namespace bo
