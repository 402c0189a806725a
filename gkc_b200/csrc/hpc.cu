// Homopolymer compression (HPC): collapse maximal runs of equal bytes in each
// read, keeping for every kept base its in-read original position
// (reference: GPU_HPCEncoding, gkc_cuda.cu:164-192, with the per-read start
// index of :180).  One warp per read: run starts by ballot, ranks by popc.
// The compacted reads form a new contiguous CSR.
#include "common.cuh"
#include "ctx.h"
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

#define CK(call)                                  \
  do {                                            \
    gkc_status _s = ctx_cuda(c, (call), #call);   \
    if (_s != GKC_OK) return _s;                  \
  } while (0)

// Homopolymer compression alone: d_out_reads gets the compressed reads back
// to back, d_out_offs[n_reads+1] their CSR offsets (from 0), d_orig_pos (may
// be NULL) the in-read position of the first base of every run.
gkc_status gkc_hpc_device(gkc_ctx *c, const char *d_reads, uint64_t n_bytes, const uint64_t *d_offs,
                          uint64_t n_reads, char *d_out_reads, uint64_t *d_out_offs,
                          int32_t *d_orig_pos) {
  using namespace gkc;
  if (!c) return GKC_ERR_INVALID_ARG;
  if (!d_offs || !d_out_offs || (n_bytes && (!d_reads || !d_out_reads)))
    return ctx_fail(c, GKC_ERR_INVALID_ARG, "null input or output");
  cudaSetDevice(c->dev);
  uint64_t ends[2] = {0, 0};
  CK(cudaMemcpyAsync(&ends[0], d_offs, 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(&ends[1], d_offs + n_reads, 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (ends[0] > ends[1] || ends[1] > n_bytes)
    return ctx_fail(c, GKC_ERR_INVALID_ARG, "read offsets decrease or pass n_bytes");
  gkc_status s;
  unsigned long long *runlen = (unsigned long long *)ws_get(c, "hpc_runlen", 8 * (n_reads + 1), &s);
  if (s != GKC_OK) return s;
  uint64_t *stmp = (uint64_t *)ws_get(c, "hpc_scan_tmp", 8 * (scan_u64_tmp_words(n_reads + 1) + 8), &s);
  if (s != GKC_OK) return s;
  const uint8_t *src = reinterpret_cast<const uint8_t *>(d_reads);
  k_hpc_count<<<c->n_sms * 8, 256, 0, c->st>>>(src, d_offs, n_reads, runlen);
  scan_u64(runlen, d_out_offs, n_reads, stmp, c->st);
  k_hpc_write<<<c->n_sms * 8, 256, 0, c->st>>>(src, d_offs, n_reads, d_out_offs,
                                               reinterpret_cast<uint8_t *>(d_out_reads), d_orig_pos);
  CK(cudaPeekAtLastError());
  CK(cudaStreamSynchronize(c->st));
  return GKC_OK;
}
