// Device-wide exclusive scan of 64-bit counters: out[i] = sum(in[0, i)),
// out[n] = total.  Reduce -> scan of tile sums -> apply (three launches).
#include "common.cuh"
#include "kernels.h"

namespace gkc {

constexpr int SCAN_NT = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_NT * SCAN_ITEMS;

__global__ void k_scan_reduce(const unsigned long long *in, uint64_t n, uint64_t *tile_sum) {
  __shared__ uint64_t tmp[32];
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
  uint64_t s = 0;
  for (int t = 0; t < SCAN_ITEMS; t++) {
    uint64_t i = base + (uint64_t)t * SCAN_NT + threadIdx.x;
    if (i < n) s += in[i];
  }
  s = block_sum_u64<SCAN_NT>(s, tmp);
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = s;
}

// single CTA: exclusive scan of the tile sums in place
__global__ void k_scan_tiles(uint64_t *tile_sum, uint64_t n_tiles) {
  __shared__ uint64_t carry;
  __shared__ uint64_t wsum[SCAN_NT / 32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint64_t b0 = 0; b0 < n_tiles; b0 += SCAN_NT) {
    uint64_t i = b0 + threadIdx.x;
    uint64_t v = i < n_tiles ? tile_sum[i] : 0, x = v;
    for (int d = 1; d < 32; d <<= 1) {
      uint64_t y = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= d) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint64_t r = 0;
      for (int w = 0; w < SCAN_NT / 32; w++) {
        uint64_t t = wsum[w];
        wsum[w] = r;
        r += t;
      }
    }
    __syncthreads();
    uint64_t excl = carry + wsum[warp] + x - v;
    __syncthreads();
    if (i < n_tiles) tile_sum[i] = excl;
    if (threadIdx.x == SCAN_NT - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) tile_sum[n_tiles] = carry;
}

__global__ void k_scan_apply(const unsigned long long *in, uint64_t n, const uint64_t *tile_sum,
                             uint64_t *out) {
  __shared__ uint64_t wsum[SCAN_NT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
  uint64_t v[SCAN_ITEMS], s = 0;
  for (int t = 0; t < SCAN_ITEMS; t++) {
    uint64_t i = base + t;
    v[t] = i < n ? in[i] : 0;
    s += v[t];
  }
  uint64_t x = s;
  for (int d = 1; d < 32; d <<= 1) {
    uint64_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t r = 0;
    for (int w = 0; w < SCAN_NT / 32; w++) {
      uint64_t t = wsum[w];
      wsum[w] = r;
      r += t;
    }
  }
  __syncthreads();
  uint64_t run = tile_sum[blockIdx.x] + wsum[warp] + x - s;
  for (int t = 0; t < SCAN_ITEMS; t++) {
    uint64_t i = base + t;
    if (i < n) out[i] = run;
    run += v[t];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
    // total, written by the last tile (its tile_sum prefix + its sum)
  }
}

__global__ void k_scan_total(const uint64_t *tile_sum, uint64_t n_tiles, uint64_t n, uint64_t *out) {
  out[n] = tile_sum[n_tiles];
}

size_t scan_u64_tmp_words(uint64_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 2; }

// Same scan over a device-side length n = min(*n_dev, n_cap): blocks past it
// contribute zero, out[n] receives the total.
__global__ void k_scan_reduce_dev(const unsigned long long *in, uint64_t n_cap, const uint64_t *n_dev,
                                  uint64_t *tile_sum) {
  __shared__ uint64_t tmp[32];
  const uint64_t n = min(n_cap, *n_dev);
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
  uint64_t s = 0;
  for (int t = 0; t < SCAN_ITEMS; t++) {
    uint64_t i = base + (uint64_t)t * SCAN_NT + threadIdx.x;
    if (i < n) s += in[i];
  }
  s = block_sum_u64<SCAN_NT>(s, tmp);
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = s;
}

__global__ void k_scan_apply_dev(const unsigned long long *in, uint64_t n_cap, const uint64_t *n_dev,
                                 const uint64_t *tile_sum, uint64_t *out) {
  const uint64_t n = min(n_cap, *n_dev);
  if ((uint64_t)blockIdx.x * SCAN_TILE >= n) return;
  __shared__ uint64_t wsum[SCAN_NT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
  uint64_t v[SCAN_ITEMS], s = 0;
  for (int t = 0; t < SCAN_ITEMS; t++) {
    uint64_t i = base + t;
    v[t] = i < n ? in[i] : 0;
    s += v[t];
  }
  uint64_t x = s;
  for (int d = 1; d < 32; d <<= 1) {
    uint64_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t r = 0;
    for (int w = 0; w < SCAN_NT / 32; w++) {
      uint64_t t = wsum[w];
      wsum[w] = r;
      r += t;
    }
  }
  __syncthreads();
  uint64_t run = tile_sum[blockIdx.x] + wsum[warp] + x - s;
  for (int t = 0; t < SCAN_ITEMS; t++) {
    uint64_t i = base + t;
    if (i < n) out[i] = run;
    run += v[t];
  }
}

__global__ void k_scan_total_dev(const uint64_t *tile_sum, uint64_t n_tiles, uint64_t n_cap,
                                 const uint64_t *n_dev, uint64_t *out) {
  out[min(n_cap, *n_dev)] = tile_sum[n_tiles];
}

void scan_u64_dev(const unsigned long long *in, uint64_t *out, uint64_t n_cap, const uint64_t *n_dev,
                  uint64_t *block_tmp, cudaStream_t st) {
  uint64_t n_tiles = (n_cap + SCAN_TILE - 1) / SCAN_TILE;
  if (n_tiles == 0) n_tiles = 1;
  k_scan_reduce_dev<<<(unsigned)n_tiles, SCAN_NT, 0, st>>>(in, n_cap, n_dev, block_tmp);
  k_scan_tiles<<<1, SCAN_NT, 0, st>>>(block_tmp, n_tiles);
  k_scan_apply_dev<<<(unsigned)n_tiles, SCAN_NT, 0, st>>>(in, n_cap, n_dev, block_tmp, out);
  k_scan_total_dev<<<1, 1, 0, st>>>(block_tmp, n_tiles, n_cap, n_dev, out);
}

void scan_u64(const unsigned long long *in, uint64_t *out, uint64_t n, uint64_t *block_tmp,
              cudaStream_t st) {
  uint64_t n_tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (n_tiles == 0) n_tiles = 1;
  k_scan_reduce<<<(unsigned)n_tiles, SCAN_NT, 0, st>>>(in, n, block_tmp);
  k_scan_tiles<<<1, SCAN_NT, 0, st>>>(block_tmp, n_tiles);
  k_scan_apply<<<(unsigned)n_tiles, SCAN_NT, 0, st>>>(in, n, block_tmp, out);
  k_scan_total<<<1, 1, 0, st>>>(block_tmp, n_tiles, n, out);
}

}  // namespace gkc
