// Checks the 16-byte SWAR comment search of csrc/q13_search.cuh (compiled
// for the host) against a byte-serial restatement of find_substring /
// matches_pattern (bespoke_tpch/query_q13.cpp:44-83) on random slices with
// small alphabets (many candidate bytes), random offsets and words of length
// 0..4, bytes past the comment differing from it.  Exit status 0 = all equal.
#include <cstdio>
#include <random>

#include "q13_search.cuh"

namespace {
uint32_t serial_find(const uint8_t* s, uint32_t from, uint32_t n, const uint8_t* w, uint32_t l) {
  if (l == 0) return from;
  if (n < l) return n;
  for (uint32_t p = from; p + l <= n; ++p) {
    uint32_t k = 0;
    while (k < l && s[p + k] == w[k]) ++k;
    if (k == l) return p;
  }
  return n;
}

bool serial_match(const uint8_t* s, uint32_t n, const uint8_t* w1, uint32_t l1, const uint8_t* w2, uint32_t l2) {
  const uint32_t p1 = serial_find(s, 0, n, w1, l1);
  if (p1 == n) return false;
  return serial_find(s, p1 + l1, n, w2, l2) != n;
}
}  // namespace

int main() {
  std::mt19937 rng(1);
  alignas(16) uint8_t slice[4096 + 32];
  long checks = 0;
  for (int it = 0; it < 100000; ++it) {
    const int alpha = 1 + rng() % 4;
    for (auto& b : slice) b = static_cast<uint8_t>('a' + rng() % alpha);
    const int s = rng() % 200, n = rng() % 90;
    uint8_t w1[8], w2[8];
    const int l1 = rng() % 5, l2 = rng() % 5;
    for (int k = 0; k < l1; ++k) w1[k] = static_cast<uint8_t>('a' + rng() % alpha);
    for (int k = 0; k < l2; ++k) w2[k] = static_cast<uint8_t>('a' + rng() % alpha);
    if (rng() % 2)
      for (int k = s + n; k < s + n + 32; ++k) slice[k] = static_cast<uint8_t>('a' + rng() % alpha);
    const bool a = bo::q13_match_slice(slice, s, n, w1, l1, w2, l2);
    const bool b = serial_match(slice + s, static_cast<uint32_t>(n), w1, l1, w2, l2);
    if (a != b) {
      std::printf("match differs: it=%d s=%d n=%d l1=%d l2=%d swar=%d serial=%d\n", it, s, n, l1, l2, a, b);
      return 1;
    }
    for (int lo = s; l1 > 0 && lo <= s + n; lo += 7) {
      const int f = bo::q13_find_slice(slice, lo, s + n, w1, l1);
      const uint32_t r = serial_find(slice, static_cast<uint32_t>(lo), static_cast<uint32_t>(s + n), w1, l1);
      if (f != (r == static_cast<uint32_t>(s + n) ? -1 : static_cast<int>(r))) {
        std::printf("find differs: it=%d lo=%d\n", it, lo);
        return 1;
      }
    }
    ++checks;
  }
  std::printf("ok %ld\n", checks);
  return 0;
}
