// Onesweep LSD radix sort (device-wide) interface.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

namespace gkc {

struct OnesweepScratch {
  unsigned long long *hist;      // 16 * 256
  unsigned long long *lookback;  // onesweep_lookback_words(n_max)
  unsigned long long *ticket;    // 1
  uint32_t *err;
  int max_ctas;
};
struct OnesweepStatus {
  int result_in_alt;  // 1 if the sorted keys ended in `alt`
};
size_t onesweep_lookback_words(uint64_t n_max);
template <typename K>
OnesweepStatus onesweep_sort(K *keys, K *alt, const uint64_t *n_dev, uint64_t n_max, int key_bits,
                             OnesweepScratch s, cudaStream_t st, uint32_t *launches);
// The same, moving a uint32 value with each key (stable: equal keys keep
// their input order, values included).
template <typename K>
OnesweepStatus onesweep_sort_kv(K *keys, K *alt, uint32_t *vals, uint32_t *valt, const uint64_t *n_dev,
                                uint64_t n_max, int key_bits, OnesweepScratch s, cudaStream_t st,
                                uint32_t *launches);

}  // namespace gkc
