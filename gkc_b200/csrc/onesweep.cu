// Device-wide LSD radix sort, onesweep form (Adinets & Merrill, "Onesweep: a
// faster least significant digit radix sort for GPUs", 2022): one upfront
// pass histograms every digit position, then each digit pass is a single
// kernel in which a tile ranks its keys stably, publishes its per-digit
// counts, and finds the counts of all earlier tiles by a decoupled
// look-back, so keys are scattered in one read and one write per pass.
//
// Keys: uint64 or unsigned __int128, sorted on their low `key_bits` bits,
// 8-bit digits.  Every wait on another tile is bounded.
#include "common.cuh"
#include "onesweep.h"

namespace gkc {

constexpr int OS_NT = 256;
constexpr int OS_ITEMS = 16;
constexpr int OS_TILE = OS_NT * OS_ITEMS;
constexpr int OS_WARPS = OS_NT / 32;
constexpr int OS_RADIX = 256;

constexpr unsigned long long OS_AGG = 1ull << 62, OS_PRE = 2ull << 62;
constexpr unsigned long long OS_VAL = (1ull << 62) - 1;

GKC_DEV unsigned long long os_ld_acquire(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
GKC_DEV void os_st_release(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

template <typename K>
GKC_DEV uint32_t os_digit(K x, int pass) {
  return (uint32_t)(x >> (8 * pass)) & 0xFFu;
}

// hist[pass][digit] over all keys, for every pass.
template <typename K>
__global__ void __launch_bounds__(OS_NT) k_os_histogram(const K *keys, const uint64_t *n_dev,
                                                        int passes, unsigned long long *hist) {
  __shared__ uint32_t h[16][OS_RADIX];
  const uint64_t n = *n_dev;
  for (int i = threadIdx.x; i < passes * OS_RADIX; i += OS_NT) h[i / OS_RADIX][i % OS_RADIX] = 0;
  __syncthreads();
  for (uint64_t i = blockIdx.x * (uint64_t)OS_NT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * OS_NT) {
    K x = keys[i];
    for (int p = 0; p < passes; p++) atomicAdd(&h[p][os_digit<K>(x, p)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * OS_RADIX; i += OS_NT) {
    uint32_t v = h[i / OS_RADIX][i % OS_RADIX];
    if (v) atomicAdd(&hist[i], (unsigned long long)v);
  }
}

// exclusive scan of each pass's 256 digit counts (one CTA, one warp per pass)
__global__ void k_os_digit_offsets(unsigned long long *hist, int passes) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int p = warp; p < passes; p += blockDim.x / 32) {
    unsigned long long carry = 0;
    for (int d0 = 0; d0 < OS_RADIX; d0 += 32) {
      unsigned long long v = hist[p * OS_RADIX + d0 + lane], x = v;
      for (int s = 1; s < 32; s <<= 1) {
        unsigned long long y = __shfl_up_sync(0xffffffffu, x, s);
        if (lane >= s) x += y;
      }
      hist[p * OS_RADIX + d0 + lane] = carry + x - v;
      carry += __shfl_sync(0xffffffffu, x, 31);
    }
  }
}

// One digit pass.  With KV, a uint32 value moves with each key (vin -> vout).
template <typename K, bool KV>
__global__ void __launch_bounds__(OS_NT) k_os_pass(const K *in, K *out, const uint32_t *vin,
                                                   uint32_t *vout, const uint64_t *n_dev, int pass,
                                                   const unsigned long long *digit_base,
                                                   unsigned long long *lookback,
                                                   unsigned long long *ticket, uint32_t *err) {
  __shared__ uint32_t warp_cnt[OS_WARPS][OS_RADIX];
  __shared__ uint64_t tile_prefix[OS_RADIX];
  __shared__ uint64_t s_tile;
  const uint64_t n = *n_dev;
  const uint64_t n_tiles = (n + OS_TILE - 1) / OS_TILE;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1ull);
    for (int i = threadIdx.x; i < OS_WARPS * OS_RADIX; i += OS_NT) (&warp_cnt[0][0])[i] = 0;
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= n_tiles) break;
    // each warp owns a contiguous segment of 32 * OS_ITEMS keys; round r,
    // lane l takes key r*32 + l of that segment, so (round, lane) order is
    // the input order and the ranks below are stable
    const uint64_t seg = tile * OS_TILE + (uint64_t)warp * 32 * OS_ITEMS;
    K key[OS_ITEMS];
    uint32_t rank[OS_ITEMS];
    uint32_t val[KV ? OS_ITEMS : 1];
#pragma unroll
    for (int r = 0; r < OS_ITEMS; r++) {
      const uint64_t i = seg + (uint64_t)r * 32 + lane;
      const bool v = i < n;
      key[r] = v ? in[i] : (K)0;
      if (KV) val[KV ? r : 0] = v ? vin[i] : 0u;
      const uint32_t d = v ? os_digit<K>(key[r], pass) : 0xFFFFFFFFu;
      const uint32_t peers = __match_any_sync(0xffffffffu, d);
      const uint32_t below = __popc(peers & ((1u << lane) - 1u));
      uint32_t base = 0;
      if (v) base = warp_cnt[warp][d];
      __syncwarp();
      rank[r] = base + below;
      // the highest peer advances the warp's counter for this digit
      if (v && (peers >> lane) == 1u) warp_cnt[warp][d] = base + __popc(peers);
      __syncwarp();
    }
    __syncthreads();
    // per digit: tile count, warp prefixes; publish and look back
    {
      const int d = threadIdx.x;  // OS_NT == OS_RADIX
      uint32_t run = 0;
      for (int w = 0; w < OS_WARPS; w++) {
        uint32_t c = warp_cnt[w][d];
        warp_cnt[w][d] = run;
        run += c;
      }
      unsigned long long *lb = lookback + tile * OS_RADIX + d;
      uint64_t excl = 0;
      if (tile == 0) {
        os_st_release(lb, OS_PRE | run);
      } else {
        os_st_release(lb, OS_AGG | run);
        uint64_t j = tile - 1;
        uint32_t it = 0;
        while (true) {
          unsigned long long v = os_ld_acquire(lookback + j * OS_RADIX + d);
          unsigned long long f = v & ~OS_VAL;
          if (f == 0) {
            if (++it > (1u << 24)) {
              atomicOr(err, ERR_SPIN_TIMEOUT);
              break;
            }
            nanosleep_backoff(it);
            continue;
          }
          excl += v & OS_VAL;
          if (f == OS_PRE || j == 0) break;
          j--;
        }
        os_st_release(lb, OS_PRE | (excl + run));
      }
      tile_prefix[d] = digit_base[pass * OS_RADIX + d] + excl;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < OS_ITEMS; r++) {
      const uint64_t i = seg + (uint64_t)r * 32 + lane;
      if (i < n) {
        const uint32_t d = os_digit<K>(key[r], pass);
        const uint64_t dst = tile_prefix[d] + warp_cnt[warp][d] + rank[r];
        out[dst] = key[r];
        if (KV) vout[dst] = val[KV ? r : 0];
      }
    }
    __syncthreads();
  }
}

template <typename K, bool KV>
static OnesweepStatus onesweep_run(K *keys, K *alt, uint32_t *vals, uint32_t *valt, const uint64_t *n_dev,
                                   uint64_t n_max, int key_bits, OnesweepScratch s, cudaStream_t st,
                                   uint32_t *launches) {
  const int passes = (key_bits + 7) / 8;
  const uint64_t tiles = (n_max + OS_TILE - 1) / OS_TILE;
  cudaMemsetAsync(s.hist, 0, sizeof(unsigned long long) * 16 * OS_RADIX, st);
  unsigned grid_h = (unsigned)std::min<uint64_t>(std::max<uint64_t>(1, (n_max + OS_NT * 8 - 1) / (OS_NT * 8)), 148 * 16);
  k_os_histogram<K><<<grid_h, OS_NT, 0, st>>>(keys, n_dev, passes, s.hist);
  k_os_digit_offsets<<<1, 32 * 8, 0, st>>>(s.hist, passes);
  *launches += 2;
  K *src = keys, *dst = alt;
  uint32_t *vsrc = vals, *vdst = valt;
  for (int p = 0; p < passes; p++) {
    cudaMemsetAsync(s.lookback, 0, sizeof(unsigned long long) * (tiles + 1) * OS_RADIX, st);
    cudaMemsetAsync(s.ticket, 0, sizeof(unsigned long long), st);
    unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)s.max_ctas));
    k_os_pass<K, KV><<<grid, OS_NT, 0, st>>>(src, dst, vsrc, vdst, n_dev, p, s.hist, s.lookback,
                                              s.ticket, s.err);
    *launches += 1;
    K *t = src;
    src = dst;
    dst = t;
    uint32_t *vt = vsrc;
    vsrc = vdst;
    vdst = vt;
  }
  return OnesweepStatus{src == keys ? 0 : 1};
}

template <typename K>
OnesweepStatus onesweep_sort(K *keys, K *alt, const uint64_t *n_dev, uint64_t n_max, int key_bits,
                             OnesweepScratch s, cudaStream_t st, uint32_t *launches) {
  return onesweep_run<K, false>(keys, alt, nullptr, nullptr, n_dev, n_max, key_bits, s, st, launches);
}

template <typename K>
OnesweepStatus onesweep_sort_kv(K *keys, K *alt, uint32_t *vals, uint32_t *valt, const uint64_t *n_dev,
                                uint64_t n_max, int key_bits, OnesweepScratch s, cudaStream_t st,
                                uint32_t *launches) {
  return onesweep_run<K, true>(keys, alt, vals, valt, n_dev, n_max, key_bits, s, st, launches);
}

size_t onesweep_lookback_words(uint64_t n_max) {
  return ((n_max + OS_TILE - 1) / OS_TILE + 1) * OS_RADIX;
}

template OnesweepStatus onesweep_sort<uint64_t>(uint64_t *, uint64_t *, const uint64_t *, uint64_t,
                                                int, OnesweepScratch, cudaStream_t, uint32_t *);
template OnesweepStatus onesweep_sort<u128>(u128 *, u128 *, const uint64_t *, uint64_t, int,
                                            OnesweepScratch, cudaStream_t, uint32_t *);
template OnesweepStatus onesweep_sort_kv<uint64_t>(uint64_t *, uint64_t *, uint32_t *, uint32_t *,
                                                   const uint64_t *, uint64_t, int, OnesweepScratch,
                                                   cudaStream_t, uint32_t *);
template OnesweepStatus onesweep_sort_kv<u128>(u128 *, u128 *, uint32_t *, uint32_t *, const uint64_t *,
                                               uint64_t, int, OnesweepScratch, cudaStream_t, uint32_t *);

}  // namespace gkc
