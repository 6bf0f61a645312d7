// Substring search over a warp's shared-memory slice of order comments,
// 16 bytes per step: the candidate starts are the bytes equal to the word's
// first byte (exact SWAR zero-byte test), each candidate is verified byte by
// byte.  Same result as the byte-serial search of find_substring
// (bespoke_tpch/query_q13.cpp:44-66) over the same bytes.
#pragma once

#include <cstdint>

#ifndef __CUDACC__
#define BO_HD
#else
#define BO_HD __host__ __device__
#endif

namespace bo {

BO_HD inline int q13_ctz(uint32_t m) {
#ifdef __CUDA_ARCH__
  return __ffs(static_cast<int>(m)) - 1;
#else
  return __builtin_ctz(m);
#endif
}

// Bit b (0..3) set where byte b of x equals the byte replicated in c4.
BO_HD inline uint32_t q13_eq_nibble(uint32_t x, uint32_t c4) {
  const uint32_t y = x ^ c4;  // zero bytes where equal
  const uint32_t t = ((y & 0x7f7f7f7fu) + 0x7f7f7f7fu) | y;
  const uint32_t z = ~t & 0x80808080u;  // 0x80 exactly in the zero bytes
  return (z * 0x00204081u) >> 28;        // bits 7, 15, 23, 31 -> 28..31
}

// First p in [lo, hi - l] with slice[p, p + l) == w, else -1.  l >= 1;
// slice is 16-byte aligned and readable up to the 16-byte boundary after
// hi - l (bytes past hi are read but never matched).
BO_HD inline int q13_find_slice(const uint8_t* slice, int lo, int hi, const uint8_t* w, int l) {
  const int last = hi - l;
  if (last < lo) return -1;
  const uint32_t c4 = 0x01010101u * w[0];
  for (int c = lo & ~15; c <= last; c += 16) {
#ifdef __CUDA_ARCH__
    const uint4 v = *reinterpret_cast<const uint4*>(slice + c);
    const uint32_t x0 = v.x, x1 = v.y, x2 = v.z, x3 = v.w;
#else
    const uint32_t* q = reinterpret_cast<const uint32_t*>(slice + c);
    const uint32_t x0 = q[0], x1 = q[1], x2 = q[2], x3 = q[3];
#endif
    uint32_t m = q13_eq_nibble(x0, c4) | (q13_eq_nibble(x1, c4) << 4) | (q13_eq_nibble(x2, c4) << 8) |
                 (q13_eq_nibble(x3, c4) << 12);
    if (c < lo) m &= 0xffffu << (lo - c);
    if (last - c < 15) m &= (2u << (last - c)) - 1u;
    while (m) {
      const int p = c + q13_ctz(m);
      m &= m - 1u;
      int k = 1;
      while (k < l && slice[p + k] == w[k]) ++k;
      if (k == l) return p;
    }
  }
  return -1;
}

// matches_pattern (query_q13.cpp:68-83) for the comment slice[s, s + n): the
// first occurrence p1 of w1 (an empty w1 at 0; none: no match), then w2 from
// p1 + l1 (an empty w2 at p1 + l1, which matches unless that is the end).
BO_HD inline bool q13_match_slice(const uint8_t* slice, int s, int n, const uint8_t* w1, int l1, const uint8_t* w2,
                                  int l2) {
  int p1 = 0;
  if (l1 > 0) {
    const int f = q13_find_slice(slice, s, s + n, w1, l1);
    p1 = f < 0 ? n : f - s;
  }
  if (p1 == n) return false;
  if (l2 == 0) return p1 + l1 != n;
  return q13_find_slice(slice, s + p1 + l1, s + n, w2, l2) >= 0;
}

}  // namespace bo
