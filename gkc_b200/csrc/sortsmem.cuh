// Shared-memory sort helpers used when a slice cannot be aggregated in the
// order-preserving hash table (too many distinct keys in a narrow key range).
#pragma once
#include "common.cuh"
#include "kernels.h"

namespace gkc {

// -------------------------------------------------------- shared-memory sort

constexpr int SC_NT = kSortThreads;  // 1024: one CTA per SM
constexpr int SC_DMAX = 12;           // bits per MSD counting pass
constexpr int SC_SMAX = 32;           // leaves up to this size: insertion sort
constexpr int SC_BIGMAX = 256;        // larger leaves recorded per pass
constexpr int SC_WARPMAX = 1024;      // leaves up to this size: sorted by one warp

template <typename K> struct SortCap;
template <> struct SortCap<uint64_t> { static constexpr int value = 5632; };
template <> struct SortCap<u128> { static constexpr int value = 2816; };

template <typename K>
struct SortSmem {
  K A[SortCap<K>::value];
  K B[SortCap<K>::value];
  uint32_t cnt[1 << SC_DMAX];
  uint32_t tmp[64];
  uint32_t big_s[SC_BIGMAX], big_m[SC_BIGMAX];
  uint32_t n_big;
  uint32_t D;
  uint64_t bucket, excl, n, start;
  // oversized-bucket frames
  struct Frame {
    uint64_t off, len;
    int skip, src, split, d;
    uint32_t cursor;
  } fr[24];
  int depth;
  int act;              // action decided by thread 0 for the oversize walk
  uint64_t c_off, c_len;
  int c_skip, c_src;
  uint64_t out;
};

template <typename K> int sort_count_cap() { return SortCap<K>::value; }
template <typename K> size_t sort_count_smem_bytes() { return sizeof(SortSmem<K>); }
template int sort_count_cap<uint64_t>();
template int sort_count_cap<u128>();
template size_t sort_count_smem_bytes<uint64_t>();
template size_t sort_count_smem_bytes<u128>();

GKC_DEV int ceil_log2_u32(uint32_t n) { return n <= 1 ? 0 : 32 - __clz(n - 1); }

// Exclusive scan of cnt[0, nd) in place; returns the total.
GKC_DEV uint32_t scan_counters(uint32_t *cnt, uint32_t nd, uint32_t *tmp) {
  const uint32_t per = (nd + SC_NT - 1) / SC_NT;
  const uint32_t c0 = threadIdx.x * per;
  uint32_t s = 0;
  for (uint32_t j = c0; j < c0 + per && j < nd; j++) s += cnt[j];
  uint32_t total;
  uint32_t run = block_exclusive_scan<SC_NT>(s, tmp, &total);
  for (uint32_t j = c0; j < c0 + per && j < nd; j++) {
    uint32_t v = cnt[j];
    cnt[j] = run;
    run += v;
  }
  __syncthreads();
  return total;
}

// In-place ascending sort of A[0, m) with a comparator network in which every
// comparator puts the smaller key at the lower index, so indices >= m can be
// treated as +infinity (the "flip" form of bitonic sort).
template <typename K>
GKC_DEV void bitonic_sort(K *A, uint32_t m) {
  uint32_t P = 1;
  while (P < m) P <<= 1;
  for (uint32_t size = 2; size <= P; size <<= 1) {
    const uint32_t half = size >> 1;
    for (uint32_t i = threadIdx.x; i < P / 2; i += SC_NT) {
      uint32_t blk = i / half, off = i % half;
      uint32_t lo = blk * size + off, hi = blk * size + size - 1 - off;
      if (hi < m) {
        K x = A[lo], y = A[hi];
        if (y < x) { A[lo] = y; A[hi] = x; }
      }
    }
    __syncthreads();
    for (uint32_t stride = size >> 2; stride >= 1; stride >>= 1) {
      for (uint32_t i = threadIdx.x; i < P / 2; i += SC_NT) {
        uint32_t blk = i / stride, off = i % stride;
        uint32_t lo = blk * 2 * stride + off, hi = lo + stride;
        if (hi < m) {
          K x = A[lo], y = A[hi];
          if (y < x) { A[lo] = y; A[hi] = x; }
        }
      }
      __syncthreads();
    }
  }
}

// In-place ascending sort of A[0, m) by one warp (the same comparator form as
// bitonic_sort, with warp barriers between stages).
template <typename K>
GKC_DEV void warp_bitonic_keys(K *A, uint32_t m) {
  uint32_t P = 1;
  while (P < m) P <<= 1;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t size = 2; size <= P; size <<= 1) {
    const uint32_t half = size >> 1;
    for (uint32_t i = lane; i < P / 2; i += 32) {
      const uint32_t blk = i / half, off = i % half;
      const uint32_t lo = blk * size + off, hi = blk * size + size - 1 - off;
      if (hi < m) {
        const K x = A[lo], y = A[hi];
        if (y < x) {
          A[lo] = y;
          A[hi] = x;
        }
      }
    }
    __syncwarp();
    for (uint32_t stride = size >> 2; stride >= 1; stride >>= 1) {
      for (uint32_t i = lane; i < P / 2; i += 32) {
        const uint32_t blk = i / stride, off = i % stride;
        const uint32_t lo = blk * 2 * stride + off, hi = lo + stride;
        if (hi < m) {
          const K x = A[lo], y = A[hi];
          if (y < x) {
            A[lo] = y;
            A[hi] = x;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Sorts S.A[0, n) ascending; keys agree on their top `skip` bits.
template <typename K>
GKC_DEV void smem_sort(SortSmem<K> &S, uint32_t n, int key_bits, int skip) {
  const int R = key_bits - skip;
  if (n <= 1 || R <= 0) return;
  const int d = max(1, min(min(SC_DMAX, R), ceil_log2_u32(n)));
  const uint32_t nd = 1u << d;
  for (uint32_t j = threadIdx.x; j < nd; j += SC_NT) S.cnt[j] = 0;
  if (threadIdx.x == 0) S.n_big = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += SC_NT)
    atomicAdd(&S.cnt[key_digit<K>(S.A[i], key_bits, skip, d)], 1u);
  __syncthreads();
  scan_counters(S.cnt, nd, S.tmp);
  for (uint32_t i = threadIdx.x; i < n; i += SC_NT) {
    K x = S.A[i];
    uint32_t pos = atomicAdd(&S.cnt[key_digit<K>(x, key_bits, skip, d)], 1u);
    S.B[pos] = x;
  }
  __syncthreads();
  // cnt[j] is now the end of leaf j
  for (uint32_t j = threadIdx.x; j < nd; j += SC_NT) {
    uint32_t s = j ? S.cnt[j - 1] : 0u, e = S.cnt[j], m = e - s;
    if (m <= (uint32_t)SC_SMAX) {
      for (uint32_t t = 0; t < m; t++) {
        K x = S.B[s + t];
        uint32_t q = t;
        while (q > 0 && x < S.A[s + q - 1]) {
          S.A[s + q] = S.A[s + q - 1];
          q--;
        }
        S.A[s + q] = x;
      }
    } else {
      uint32_t slot = atomicAdd(&S.n_big, 1u);
      if (slot < (uint32_t)SC_BIGMAX) {
        S.big_s[slot] = s;
        S.big_m[slot] = m;
      }
    }
  }
  __syncthreads();
  const uint32_t nbig = min(S.n_big, (uint32_t)SC_BIGMAX);
  // leaves up to SC_WARPMAX keys: one warp each, all at once
  for (uint32_t t = threadIdx.x >> 5; t < nbig; t += SC_NT / 32) {
    const uint32_t s = S.big_s[t], m = S.big_m[t];
    if (m > (uint32_t)SC_WARPMAX) continue;
    for (uint32_t i = threadIdx.x & 31u; i < m; i += 32) S.A[s + i] = S.B[s + i];
    __syncwarp();
    warp_bitonic_keys<K>(S.A + s, m);
  }
  __syncthreads();
  // larger leaves: the whole block, one after another
  for (uint32_t t = 0; t < nbig; t++) {
    const uint32_t s = S.big_s[t], m = S.big_m[t];
    if (m <= (uint32_t)SC_WARPMAX) continue;
    for (uint32_t i = threadIdx.x; i < m; i += SC_NT) S.A[s + i] = S.B[s + i];
    __syncthreads();
    bitonic_sort<K>(S.A + s, m);
  }
  // big leaves beyond the list (at most n / SC_SMAX exist, so only when
  // n > SC_BIGMAX * SC_SMAX) are sorted by one more bitonic pass overall.
  if (S.n_big > (uint32_t)SC_BIGMAX) {
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nd; j += SC_NT) {
      uint32_t s = j ? S.cnt[j - 1] : 0u, e = S.cnt[j];
      if (e - s > (uint32_t)SC_SMAX)
        for (uint32_t i = s; i < e; i++) S.A[i] = S.B[i];
    }
    __syncthreads();
    bitonic_sort<K>(S.A, n);
  }
  __syncthreads();
}

// Run-length pass over sorted S.A[0, n): run starts go to S.B viewed as
// uint32 (run j spans [rs[j], rs[j+1])).  Returns the number of runs.
template <typename K>
GKC_DEV uint32_t smem_runs(SortSmem<K> &S, uint32_t n) {
  uint32_t *rs = reinterpret_cast<uint32_t *>(S.B);
  const uint32_t per = (n + SC_NT - 1) / SC_NT;
  const uint32_t c0 = threadIdx.x * per;
  uint32_t cntr = 0;
  for (uint32_t i = c0; i < c0 + per && i < n; i++) cntr += (i == 0 || S.A[i] != S.A[i - 1]);
  uint32_t total;
  uint32_t idx = block_exclusive_scan<SC_NT>(cntr, S.tmp, &total);
  for (uint32_t i = c0; i < c0 + per && i < n; i++)
    if (i == 0 || S.A[i] != S.A[i - 1]) rs[idx++] = i;
  if (threadIdx.x == 0) rs[total] = n;
  __syncthreads();
  return total;
}

template <typename K>
GKC_DEV void write_runs(SortSmem<K> &S, uint32_t D, K *out_keys, uint32_t *out_counts,
                        uint64_t out) {
  const uint32_t *rs = reinterpret_cast<const uint32_t *>(S.B);
  for (uint32_t j = threadIdx.x; j < D; j += SC_NT) {
    out_keys[out + j] = S.A[rs[j]];
    out_counts[out + j] = rs[j + 1] - rs[j];
  }
}

template <typename K>
GKC_DEV void load_keys(K *dst, const K *src, uint32_t n) {
  for (uint32_t i = threadIdx.x; i < n; i += SC_NT) dst[i] = src[i];
}

}  // namespace gkc
