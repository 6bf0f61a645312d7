// Shared device helpers for the bespoke GPU engine (sm_100a only).
//
// Everything on the hot path is integer / fixed-point arithmetic: the reference
// pipelines (bespoke_tpch/query_q1.cpp:27-34, query_q3.cpp:219-260) keep decimal
// sums in int64 / __int128, so every aggregate here is exact.  128-bit totals are
// accumulated in global memory as two 64-bit words with an explicit carry
// (atomic_add_i128), because the hardware has no 128-bit atomic add.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "bespoke_gpu.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "bespoke GPU kernels are written for sm_100a (B200) only"
#endif

namespace bo {

// Device-side error bits, OR-ed into the context's error word by kernels and
// translated into status codes by the host after the pipeline's single sync.
enum : uint32_t {
  kErrBadGroupCode = 1u << 0,   // a row's group code is outside the declared domain
  kErrValueRange = 1u << 1,     // a value outside the exact-arithmetic contract
  kErrTableOverflow = 1u << 2,  // a hash / group table ran past its capacity
  kErrSpinTimeout = 1u << 3,    // a bounded device-side wait gave up
  kErrOutputOverflow = 1u << 4, // an output buffer was too small
  kErrSumOverflow = 1u << 5,    // a 128-bit total does not fit the 64-bit result field
};

// ------------------------------------------- programmatic dependent launch --
// A kernel launched with the programmatic-serialization attribute may start
// while the kernel before it on the stream still runs.  pdl_wait() blocks
// until that kernel has completed and its writes are visible (a no-op for a
// kernel launched the ordinary way); pdl_launch_dependents() lets the next
// such kernel be scheduled once every block of this one has issued it.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }

// ---------------------------------------------------------------- loads ----
// Streaming 128-bit loads: read-only, not allocated in L1 (each byte of a fact
// column is touched exactly once per scan).
__device__ __forceinline__ int4 ld_stream_v4(const void* p) {
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}
__device__ __forceinline__ uint2 ld_stream_v2(const void* p) {
  uint2 v;
  asm volatile("ld.global.nc.L1::no_allocate.v2.u32 {%0,%1}, [%2];"
               : "=r"(v.x), "=r"(v.y)
               : "l"(p));
  return v;
}
__device__ __forceinline__ uint32_t ld_stream_u32(const void* p) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// 256-bit streaming loads (sm_100): one full 32-byte sector per lane per
// instruction, so a warp consumes whole sectors whatever its lane stride.
struct int8v {
  int v[8];
};
__device__ __forceinline__ int8v ld_stream_v8(const void* p) {
  int8v r;
  asm volatile("ld.global.nc.L1::no_allocate.v8.s32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
                 "=r"(r.v[6]), "=r"(r.v[7])
               : "l"(p));
  return r;
}
// The same 256-bit streaming load, marked evict-first in L2: for a column
// scanned once alongside lookups into structures that should stay in L2 (hash
// tables, bitmaps, filters), so the stream does not push them out.
__device__ __forceinline__ int8v ld_first_v8(const void* p) {
  int8v r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::evict_first.v8.s32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
                 "=r"(r.v[6]), "=r"(r.v[7])
               : "l"(p));
  return r;
}
struct long4v {
  long long v[4];
};
__device__ __forceinline__ long4v ld_stream_v4x64(const void* p) {
  long4v r;
  asm volatile("ld.global.nc.L1::no_allocate.v4.s64 {%0,%1,%2,%3}, [%4];"
               : "=l"(r.v[0]), "=l"(r.v[1]), "=l"(r.v[2]), "=l"(r.v[3])
               : "l"(p));
  return r;
}

__device__ __forceinline__ int64_t make_i64(int lo, int hi) {
  return (int64_t)(((uint64_t)(uint32_t)hi << 32) | (uint32_t)lo);
}

// ------------------------------------------------------- 128-bit totals ----
// Adds a signed 128-bit value into a {lo, hi} pair of 64-bit words.  The carry
// out of each individual low-word addition is exactly determined by the old
// value the atomic returns, so the sum of all carries equals the true carry and
// the final pair is exact modulo 2^128 regardless of interleaving.
__device__ __forceinline__ void atomic_add_i128(unsigned long long* lo_hi, __int128 v) {
  const unsigned long long add_lo = (unsigned long long)(uint64_t)v;
  const unsigned long long add_hi = (unsigned long long)(uint64_t)(v >> 64);
  const unsigned long long old = atomicAdd(lo_hi, add_lo);
  const unsigned long long carry = (old + add_lo) < old ? 1ull : 0ull;
  const unsigned long long hi = add_hi + carry;
  if (hi != 0ull) atomicAdd(lo_hi + 1, hi);
}

__device__ __forceinline__ int64_t warp_sum_i64(int64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ uint32_t warp_sum_u32(uint32_t v) {
  return __reduce_add_sync(0xffffffffu, v);
}

__device__ __forceinline__ void raise_error(uint32_t* err, uint32_t bits) {
  if (err) atomicOr(err, bits);
}

// --------------------------------------------------------- bounded waits ----
// Global nanosecond timer; every spin in this library is bounded by it so a wait
// that can never complete turns into an error bit instead of a hung GPU.
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_acquire_u64(const unsigned long long* p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Hash for 32-bit join / group keys (murmur3 finaliser; any good 32-bit mixer
// works, the tables only need the low bits to be well spread).
__device__ __host__ __forceinline__ uint32_t hash32(uint32_t k) {
  k ^= k >> 16;
  k *= 0x85ebca6bu;
  k ^= k >> 13;
  k *= 0xc2b2ae35u;
  k ^= k >> 16;
  return k;
}

// --------------------------------------------------- 128-bit helpers ------
__device__ __forceinline__ __int128 load_i128(const unsigned long long* p) {
  const uint64_t lo = __ldcg(p), hi = __ldcg(p + 1);
  return (__int128)(((unsigned __int128)hi << 64) | lo);
}

__device__ __forceinline__ int64_t narrow_i64(__int128 v, uint32_t& bad) {
  if (v != (__int128)(int64_t)v) bad |= kErrSumOverflow;
  return (int64_t)v;
}

__host__ __device__ __forceinline__ bo_i128 to_bo_i128(__int128 v) {
  bo_i128 r;
  r.lo = (uint64_t)v;
  r.hi = (int64_t)(v >> 64);
  return r;
}

// Sum of an unsigned 128-bit value over the block, returned in thread 0.
// `scratch` holds blockDim.x + 32 entries.  Warp leaders add their warp's
// values serially in 128 bits, thread 0 adds the warp totals: exact for any
// inputs, and cheap because it runs once per block.
__device__ __forceinline__ unsigned __int128 block_sum_u128(unsigned __int128 v, unsigned __int128* scratch) {
  scratch[threadIdx.x] = v;
  __syncthreads();
  const int nw = (int)(blockDim.x >> 5);
  if ((threadIdx.x & 31) == 0) {
    unsigned __int128 t = 0;
    for (int i = 0; i < 32; ++i) t += scratch[threadIdx.x + i];
    scratch[blockDim.x + (threadIdx.x >> 5)] = t;
  }
  __syncthreads();
  unsigned __int128 tot = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < nw; ++w) tot += scratch[blockDim.x + w];
  __syncthreads();
  return tot;
}

// Last-block epilogue: true in every thread of the block that finished last
// (all other blocks' global atomics are then visible to it).
__device__ __forceinline__ bool last_block(uint32_t* done, uint32_t blocks) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) is_last = (atomicAdd(done, 1u) == blocks - 1);
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

__device__ __forceinline__ bool last_block(uint32_t* done) { return last_block(done, gridDim.x); }

// ------------------------------------------- TMA bulk copies (no multicast) --
// One-shot global -> shared bulk copy completed on an mbarrier.  Only this
// CTA's shared memory and this GPU's global memory are involved.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false if the phase did not complete within limit_ns.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
  }
  return true;
}

constexpr uint64_t kWaitLimitNs = 1000000000ull;  // 1 s bound on any device-side wait

}  // namespace bo
