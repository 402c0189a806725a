// Homopolymer compression (HPC): collapse maximal runs of equal bytes in each
// read, keeping for every kept base its in-read original position
// (reference: GPU_HPCEncoding, gkc_cuda.cu:164-192, with the per-read start
// index of :180).  One warp per read: run starts by ballot, ranks by popc.
// The compacted reads form a new contiguous CSR.
#include "common.cuh"
#include "kernels.h"

namespace gkc {

__global__ void k_hpc_count(const uint8_t *reads, const uint64_t *offs, uint64_t n_reads,
                            unsigned long long *run_len) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  for (uint64_t r = warp; r < n_reads; r += nwarps) {
    const uint64_t b = offs[r], e = offs[r + 1];
    uint32_t cnt = 0;
    for (uint64_t i0 = b; i0 < e; i0 += 32) {
      uint64_t i = i0 + lane;
      bool f = i < e && (i == b || reads[i] != reads[i - 1]);
      cnt += __popc(__ballot_sync(0xffffffffu, f));
    }
    if (lane == 0) run_len[r] = cnt;
  }
}

__global__ void k_hpc_write(const uint8_t *reads, const uint64_t *offs, uint64_t n_reads,
                            const uint64_t *hpc_offs, uint8_t *out, int32_t *orig_pos) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  for (uint64_t r = warp; r < n_reads; r += nwarps) {
    const uint64_t b = offs[r], e = offs[r + 1];
    uint64_t pos = hpc_offs[r];
    for (uint64_t i0 = b; i0 < e; i0 += 32) {
      uint64_t i = i0 + lane;
      bool f = i < e && (i == b || reads[i] != reads[i - 1]);
      uint32_t m = __ballot_sync(0xffffffffu, f);
      if (f) {
        uint64_t q = pos + __popc(m & ((1u << lane) - 1u));
        out[q] = reads[i];
        if (orig_pos) orig_pos[q] = (int32_t)(i - b);
      }
      pos += __popc(m);
    }
  }
}

}  // namespace gkc
