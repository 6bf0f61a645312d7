// Device helpers shared by the CEB pipelines (the reference's CEB engine,
// bespoke_ceb/): null tests on the column layout, warp-aggregated list
// appends, id masks of dimension tables and the ILIKE matcher.
#pragma once

#include "common.cuh"

namespace bo {

constexpr int kCebBlock = 256;

__device__ __forceinline__ bool ceb_null(const bo_ceb_col& c, int64_t r) { return c.is_null && c.is_null[r]; }

// Appends v to list[] with one reservation per warp (the lanes whose `take`
// holds).  Every lane of the warp must call it.
template <class T, class Count = unsigned int>
__device__ __forceinline__ void warp_append(bool take, const T& v, T* __restrict__ list, Count* __restrict__ count) {
  const unsigned int mask = __ballot_sync(0xffffffffu, take);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  Count base = 0;
  if (lane == leader) base = atomicAdd(count, (Count)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (take) list[base + __popc(mask & ((1u << lane) - 1u))] = v;
}

// match[c] = whether dictionary string c matches the ILIKE pattern (one
// thread per distinct string).
__global__ void ceb_like_dict_kernel(const char* __restrict__ bytes, const uint32_t* __restrict__ off, int64_t n,
                                     int32_t type, const char* __restrict__ pat, int32_t len,
                                     uint8_t* __restrict__ match);

// mask[id] = 1 for the dimension rows with a non-null id in [0, mask_size)
// and a non-null string whose code is allowed (the reference's
// build_id_mask_from_dim / build_allowed_id_mask, bespoke_ceb/query_q1a.cpp:
// 93-117, query_q10a.cpp:284-309).
__global__ void __launch_bounds__(kCebBlock) ceb_dim_mask_kernel(bo_ceb_col id, bo_ceb_col code, int64_t n,
                                                                 const uint8_t* __restrict__ allowed, int32_t n_codes,
                                                                 int32_t mask_size, uint8_t* __restrict__ mask,
                                                                 unsigned int* __restrict__ any);

// Exclusive scan of n uint32 counts into out[0..n] (out[n] = the total), on
// the context's stream: per-tile sums, their scan in one block, then each
// tile's scan plus its base.
int ceb_exclusive_scan(bo_ctx* ctx, const unsigned int* in, int64_t n, unsigned int* out);

// ILIKE on lower-cased text, the reference's LikePattern kinds
// (bespoke_ceb/query_q10a.cpp:73-246): the text is lower-cased byte by byte
// (A-Z only, as std::tolower in the C locale) while it is matched.
enum CebLike : int32_t { kLikeAll = 0, kLikeExact = 1, kLikePrefix = 2, kLikeSuffix = 3, kLikeContains = 4,
                         kLikeGeneral = 5 };

__device__ __forceinline__ char ceb_lower(char c) { return (c >= 'A' && c <= 'Z') ? (char)(c + 32) : c; }

__device__ __forceinline__ bool ceb_like_general(const char* pat, int plen, const char* s, int n) {
  int p = 0, t = 0, star = -1, match = 0;
  while (t < n) {
    const char c = ceb_lower(s[t]);
    if (p < plen && (pat[p] == '_' || pat[p] == c)) {
      ++p;
      ++t;
      continue;
    }
    if (p < plen && pat[p] == '%') {
      star = p++;
      match = t;
      continue;
    }
    if (star >= 0) {
      p = star + 1;
      t = ++match;
      continue;
    }
    return false;
  }
  while (p < plen && pat[p] == '%') ++p;
  return p == plen;
}

__device__ __forceinline__ bool ceb_like(int32_t type, const char* tok, int tlen, const char* s, int n) {
  switch (type) {
    case kLikeAll:
      return true;
    case kLikeExact:
    case kLikePrefix:
      if (type == kLikeExact ? n != tlen : n < tlen) return false;
      for (int i = 0; i < tlen; ++i)
        if (ceb_lower(s[i]) != tok[i]) return false;
      return true;
    case kLikeSuffix:
      if (n < tlen) return false;
      for (int i = 0; i < tlen; ++i)
        if (ceb_lower(s[n - tlen + i]) != tok[i]) return false;
      return true;
    case kLikeContains:
      if (tlen == 0) return true;
      for (int st = 0; st + tlen <= n; ++st) {
        int j = 0;
        while (j < tlen && ceb_lower(s[st + j]) == tok[j]) ++j;
        if (j == tlen) return true;
      }
      return false;
    default:
      return ceb_like_general(tok, tlen, s, n);
  }
}

}  // namespace bo
