// Shared device helpers for the GKC partition-and-count kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

typedef unsigned __int128 u128;

#define GKC_DEV __device__ __forceinline__

namespace gkc {

// Device error word bits (read back by the host after a pipeline run).
enum : uint32_t {
  ERR_SPIN_TIMEOUT = 1u << 0,   // a bounded wait ran out (look-back / tile chain)
  ERR_CAPACITY = 1u << 1,       // an output buffer sized in advance was too small
  ERR_OVERSIZE_SCRATCH = 1u << 2,
  ERR_BAD_READ = 1u << 3,       // a read longer than the supported superkmer length
  ERR_BOUNDS = 1u << 4,         // a device bounds check failed (access skipped)
  ERR_BIN_TOO_LARGE = 1u << 5,  // a bin holds 2^32 or more k-mers
};

// Bounded spin limit for any wait on another CTA (~0.5-2 s with backoff).
constexpr uint32_t kSpinLimit = 1u << 22;

// ASCII -> 2-bit code with the reference's mapping (A/a/U/u 0, C/c 1, G/g 2,
// T/t 3, anything else 255), built once into shared memory per CTA.
GKC_DEV uint32_t code_of_byte(uint32_t c) {
  uint32_t u = c & 0xDFu;  // fold lower case
  if (c >= 0x80u) return 255u;
  if (u == 'A' || u == 'U') return 0u;
  if (u == 'C') return 1u;
  if (u == 'G') return 2u;
  if (u == 'T') return 3u;
  return 255u;
}

// Which p-mers may be minimizers (the reference selects one at compile time,
// FILTER_KERNEL, gkc_cuda.cu:6, from the variants at :196-227):
//   0 new_filter2 (the reference's choice): the top three bases of the p-mer
//     value are not AAA, ACA or AGA;
//   1 every p-mer (its mm_filter);
//   2 new_filter: the second and third bases from the top are not both A;
//   3 sign_filter (KMC2 signatures): no AA in the lowest p-1 bases, and the
//     top three bases are not AAA or ACA.
// Values are taken unmasked, as the reference does.
enum : int { FILTER_NEW2 = 0, FILTER_ALL = 1, FILTER_NEW = 2, FILTER_SIGNATURE = 3 };

GKC_DEV bool mm_filter(uint32_t v, int p, int filter = FILTER_NEW2) {
  const uint32_t t = v >> (2 * (p - 3));
  switch (filter) {
    case FILTER_ALL:
      return true;
    case FILTER_NEW:
      return (((v >> (2 * (p - 2))) & 3u) + ((v >> (2 * (p - 3))) & 3u)) != 0u;
    case FILTER_SIGNATURE: {
      uint32_t x = v;
      bool ok = true;
      for (int i = 0; i < p - 2; i++) {
        ok &= (x & 0xFu) != 0u;
        x >>= 2;
      }
      return ok & (t != 0u) & (t != 4u);
    }
    default:
      return (t != 0u) & (t != 4u) & (t != 8u);
  }
}

// Reverse complement of a 2k-bit k-mer held in the low bits of x.
GKC_DEV uint64_t revcomp64(uint64_t x, int k) {
  x = ~x;
  x = __brevll(x);                                              // reverse bit order
  x = ((x >> 1) & 0x5555555555555555ULL) | ((x & 0x5555555555555555ULL) << 1);  // re-pair
  return x >> (64 - 2 * k);
}

GKC_DEV u128 revcomp128(u128 x, int k) {
  uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
  uint64_t rlo = revcomp64(hi, 32), rhi = revcomp64(lo, 32);  // full 128-bit revcomp
  u128 r = ((u128)rhi << 64) | rlo;
  return r >> (128 - 2 * k);
}

template <typename K>
GKC_DEV K revcomp_k(K x, int k);
template <>
GKC_DEV uint64_t revcomp_k<uint64_t>(uint64_t x, int k) { return revcomp64(x, k); }
template <>
GKC_DEV u128 revcomp_k<u128>(u128 x, int k) { return revcomp128(x, k); }

template <typename K>
GKC_DEV K kmer_mask(int k) {
  return (2 * k >= (int)(8 * sizeof(K))) ? ~(K)0 : (((K)1 << (2 * k)) - 1);
}

// Top `nbits` bits of a 2k-bit key, below the `skip` most significant bits.
template <typename K>
GKC_DEV uint32_t key_digit(K x, int key_bits, int skip, int nbits) {
  if (nbits <= 0) return 0u;
  int sh = key_bits - skip - nbits;
  return (uint32_t)(x >> sh) & ((1u << nbits) - 1u);
}

GKC_DEV uint32_t lane_id() { return threadIdx.x & 31u; }

// Block-wide exclusive scan of one uint32 per thread; returns the exclusive
// prefix and writes the block total to *total.  `tmp` holds >= 33 words.
template <int NT>
GKC_DEV uint32_t block_exclusive_scan(uint32_t v, uint32_t *tmp, uint32_t *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) tmp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = (lane < NT / 32) ? tmp[lane] : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += y;
    }
    tmp[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  uint32_t warp_prefix = warp ? tmp[warp - 1] : 0u;
  uint32_t res = warp_prefix + x - v;
  if (total) *total = tmp[NT / 32 - 1];
  __syncthreads();
  return res;
}

template <int NT>
GKC_DEV uint64_t block_sum_u64(uint64_t v, uint64_t *tmp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
  if (lane == 0) tmp[warp] = v;
  __syncthreads();
  uint64_t r = 0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < NT / 32; w++) r += tmp[w];
    tmp[0] = r;
  }
  __syncthreads();
  r = tmp[0];
  __syncthreads();
  return r;
}

GKC_DEV void nanosleep_backoff(uint32_t it) {
  if (it > 64) __nanosleep(it > 4096 ? 256 : 32);
}

}  // namespace gkc
