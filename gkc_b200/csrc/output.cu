// Count output options on the device: the frequency filter of the reference
// (kmc_counting_GPU keeps a k-mer when kmer_min_freq <= count <=
// kmer_max_freq, kmer_counting.cu:188-190, defaults utilities.hpp:109; the
// filter is commented out there) and the merged global list (one sorted list
// over all bins, with the counts of a k-mer that occurs in several bins --
// possible when reads hold N -- added up).
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "ctx.h"
#include "kernels.h"
#include "onesweep.h"

namespace gkc {

__global__ void k_keep_flags(const uint32_t *counts, uint64_t n, uint32_t lo, uint32_t hi,
                             unsigned long long *flags) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t c = counts[i];
    flags[i] = (c >= lo && c <= hi) ? 1ull : 0ull;
  }
}

template <typename K>
__global__ void k_keep_copy(const K *keys, const uint32_t *counts, const uint64_t *pos, uint64_t n, uint32_t lo,
                            uint32_t hi, K *out_keys, uint32_t *out_counts) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t c = counts[i];
    if (c >= lo && c <= hi) {
      out_keys[pos[i]] = keys[i];
      out_counts[pos[i]] = c;
    }
  }
}

// bin b of the kept list starts where bin b of the full list started
__global__ void k_keep_bins(const uint64_t *bin_off, uint32_t nbins, const uint64_t *pos, uint64_t *out) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b <= nbins; b += gridDim.x * blockDim.x)
    out[b] = pos[bin_off[b]];
}

// sum of the counts of each run of equal keys (runs start at starts[j])
__global__ void k_run_sums(const uint32_t *vals, const uint64_t *starts, uint64_t d, uint64_t n, uint32_t *out) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < d; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t e = j + 1 < d ? starts[j + 1] : n;
    uint64_t s = 0;
    for (uint64_t i = starts[j]; i < e; i++) s += vals[i];
    out[j] = s > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)s;
  }
}

}  // namespace gkc

using namespace gkc;

#define CK(call)                                  \
  do {                                            \
    gkc_status _s = ctx_cuda(c, (call), #call);   \
    if (_s != GKC_OK) return _s;                  \
  } while (0)
#define WS(ptr, type, name, count)                                      \
  type *ptr;                                                            \
  do {                                                                  \
    gkc_status _s;                                                      \
    ptr = (type *)ws_get(c, name, sizeof(type) * (size_t)(count), &_s); \
    if (_s != GKC_OK) return _s;                                        \
  } while (0)

// Keeps the entries of (keys, counts, bin_off) whose count is in [lo, hi];
// returns the kept list in the "flt_*" workspaces.
template <typename K>
static gkc_status keep_range(gkc_ctx *c, const K *keys, const uint32_t *counts, const uint64_t *bin_off,
                             uint32_t nbins, uint64_t n, uint32_t lo, uint32_t hi, uint64_t *n_out) {
  const unsigned grid = c->n_sms * 8;
  WS(flags, unsigned long long, "flt_flags", n + 1);
  WS(pos, uint64_t, "flt_pos", n + 2);
  WS(stmp, uint64_t, "flt_scan_tmp", scan_u64_tmp_words(n + 1) + 8);
  WS(ok, K, "flt_keys", n + 1);
  WS(oc, uint32_t, "flt_counts", n + 1);
  WS(ob, uint64_t, "flt_bin_off", nbins + 1);
  k_keep_flags<<<grid, 256, 0, c->st>>>(counts, n, lo, hi, flags);
  scan_u64(flags, pos, n, stmp, c->st);
  k_keep_copy<K><<<grid, 256, 0, c->st>>>(keys, counts, pos, n, lo, hi, ok, oc);
  k_keep_bins<<<(nbins + 256) / 256, 256, 0, c->st>>>(bin_off, nbins, pos, ob);
  CK(cudaPeekAtLastError());
  CK(cudaMemcpyAsync(n_out, pos + n, 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return GKC_OK;
}

template <typename K>
static gkc_status count_output_t(gkc_ctx *c, uint32_t lo, uint32_t hi, int merged, uint64_t *n_out,
                                 uint32_t *nbins_out) {
  const gkc_count_view &v = c->cv;
  const uint64_t n = v.n_distinct;
  const K *keys = reinterpret_cast<const K *>(v.keys);
  if (!merged) {
    *nbins_out = v.nbins;
    return keep_range<K>(c, keys, v.counts, v.bin_off, v.nbins, n, lo, hi, n_out);
  }
  // merged: sort (key, count) pairs by key, sum the counts of equal keys
  const unsigned grid = c->n_sms * 8;
  WS(mk, K, "merge_keys", n + 16);
  WS(mk2, K, "merge_keys_alt", n + 16);
  WS(mv, uint32_t, "merge_vals", n + 16);
  WS(mv2, uint32_t, "merge_vals_alt", n + 16);
  WS(nd, uint64_t, "merge_n", 2);
  CK(cudaMemcpyAsync(mk, keys, n * sizeof(K), cudaMemcpyDeviceToDevice, c->st));
  CK(cudaMemcpyAsync(mv, v.counts, n * 4, cudaMemcpyDeviceToDevice, c->st));
  uint64_t hn = n;
  CK(cudaMemcpyAsync(nd, &hn, 8, cudaMemcpyHostToDevice, c->st));
  WS(os_hist, unsigned long long, "merge_os_hist", 16 * 256);
  WS(os_lb, unsigned long long, "merge_os_lookback", onesweep_lookback_words(n + 1));
  WS(os_ticket, unsigned long long, "merge_os_ticket", 2);
  WS(err, uint32_t, "merge_err", 4);
  CK(cudaMemsetAsync(err, 0, 16, c->st));
  OnesweepScratch os{os_hist, os_lb, os_ticket, err, c->n_sms * 4};
  uint32_t launches = 0;
  OnesweepStatus r = onesweep_sort_kv<K>(mk, mk2, mv, mv2, nd, n, 2 * c->ck, os, c->st, &launches);
  const K *sk = r.result_in_alt ? mk2 : mk;
  const uint32_t *sv = r.result_in_alt ? mv2 : mv;
  const uint64_t nblk = rle_block_count(n);
  WS(rblk, unsigned long long, "merge_rle_blk", nblk + 1);
  WS(roff, uint64_t, "merge_rle_off", nblk + 2);
  WS(rtmp, uint64_t, "merge_rle_tmp", scan_u64_tmp_words(nblk + 1) + 8);
  WS(cur, unsigned long long, "merge_cursor", 2);
  WS(uk, K, "merge_unique_keys", n + 1);
  WS(st, uint64_t, "merge_starts", n + 1);
  WS(us, uint32_t, "merge_sums", n + 1);
  WS(bo, uint64_t, "merge_bin_off", 2);
  CK(cudaMemsetAsync(cur, 0, 16, c->st));
  rle_runs<K>(sk, n, rblk, roff, rtmp, cur, uk, st, c->st);
  uint64_t d = 0;
  uint32_t e = 0;
  if (nblk) CK(cudaMemcpyAsync(&d, roff + nblk, 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (e & ERR_SPIN_TIMEOUT) return ctx_fail(c, GKC_ERR_DEVICE_TIMEOUT, "sort look-back timed out");
  if (d) k_run_sums<<<grid, 256, 0, c->st>>>(sv, st, d, n, us);
  uint64_t hb[2] = {0, d};
  CK(cudaMemcpyAsync(bo, hb, 16, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  *nbins_out = 1;
  return keep_range<K>(c, uk, us, bo, 1, d, lo, hi, n_out);
}

gkc_status gkc_count_output(gkc_ctx *c, uint32_t min_count, uint32_t max_count, int merged, uint64_t *n_out,
                            uint64_t *bin_off, uint64_t *keys, uint32_t *counts) {
  if (!c || !n_out) return GKC_ERR_INVALID_ARG;
  if (!c->have_count) return ctx_fail(c, GKC_ERR_INVALID_ARG, "no count result in the context");
  if (min_count > max_count) return ctx_fail(c, GKC_ERR_INVALID_ARG, "min_count > max_count");
  cudaSetDevice(c->dev);
  const int kw = c->cv.key_words;
  const bool same = c->have_out && c->out_gen == c->count_gen && c->out_min == min_count &&
                    c->out_max == max_count && c->out_merged == merged;
  if (!same) {
    uint64_t n = 0;
    uint32_t nb = 0;
    gkc_status s = kw == 1 ? count_output_t<uint64_t>(c, min_count, max_count, merged, &n, &nb)
                           : count_output_t<u128>(c, min_count, max_count, merged, &n, &nb);
    if (s != GKC_OK) return s;
    c->have_out = true;
    c->out_gen = c->count_gen;
    c->out_min = min_count;
    c->out_max = max_count;
    c->out_merged = merged;
    c->out_n = n;
    c->out_nbins = nb;
  }
  *n_out = c->out_n;
  const uint64_t n = c->out_n;
  if (bin_off) CK(cudaMemcpy(bin_off, c->bufs["flt_bin_off"].p, 8 * (c->out_nbins + 1), cudaMemcpyDeviceToHost));
  if (keys && n) CK(cudaMemcpy(keys, c->bufs["flt_keys"].p, 8 * kw * n, cudaMemcpyDeviceToHost));
  if (counts && n) CK(cudaMemcpy(counts, c->bufs["flt_counts"].p, 4 * n, cudaMemcpyDeviceToHost));
  return GKC_OK;
}
