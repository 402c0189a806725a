// Per-window minimizer rules shared by the fused and the plain partition.
#pragma once
#include "common.cuh"

namespace gkc {

// Exact reference update rule for one window (gkc_cuda.cu:256-286), on codes
// that may be 255.  `code(i)` returns the code of window base i.
template <typename CodeFn>
GKC_DEV uint32_t exact_window_minimizer(CodeFn code, int k, int p, int filter = FILTER_NEW2) {
  const uint32_t M = 0xFFFFFFFFu >> (32 - 2 * p);
  uint32_t f = 0, r = 0, m, mr, best;
  for (int j = 0; j < p; j++) f = (f << 2) | code(j);
  m = mm_filter(f, p, filter) ? f : M;
  for (int j = p - 1; j >= 0; j--) {
    uint32_t c = code(j);
    r = (r << 2) | (c == 255u ? 255u : 3u - c);
  }
  mr = mm_filter(r, p, filter) ? r : M;
  best = (mr < m) ? mr : m;
  for (int j = p; j < k; j++) {
    uint32_t c = code(j);
    uint32_t cc = (c == 255u) ? 255u : 3u - c;
    f = ((f << 2) | c) & M;
    r = (r >> 2) | (cc << (2 * p - 2));
    if (mm_filter(f, p, filter)) m = f;
    if (mm_filter(r, p, filter)) mr = r;
    best = (best < m) ? best : m;
    best = (best < mr) ? best : mr;
  }
  return best;
}

GKC_DEV bool global_rs(const uint32_t *rs_bits, uint64_t pos) {
  return (rs_bits[pos >> 5] >> (pos & 31)) & 1u;
}

GKC_DEV uint32_t global_code(const uint8_t *reads, uint64_t nbytes, int64_t pos) {
  if (pos < 0 || (uint64_t)pos >= nbytes) return 255u;
  return code_of_byte(reads[pos]);
}

// Window starting at global position s: inside one read?
GKC_DEV bool global_window_valid(const uint32_t *rs_bits, uint64_t nbytes, uint64_t s, int k) {
  if (s + k > nbytes) return false;
  for (int j = 1; j < k; j++)
    if (global_rs(rs_bits, s + j)) return false;
  return true;
}

}  // namespace gkc
