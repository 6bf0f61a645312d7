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

}  // namespace bo
