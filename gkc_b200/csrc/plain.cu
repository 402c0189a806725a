// Plain per-stage form of the pipeline: the reference's stage structure on
// the device, one launch per stage, intermediates materialised in HBM.
//
// Partition (reference: GPU_GenMinimizer, GPU_GenSKM, SKMStore::add_skms;
// gkc_cuda.cu:234-324, superkmers.hpp:167-186):
//   k_plain_minimizer   one thread per window, the exact per-window rule,
//                       minimizers written to a per-position array;
//   k_plain_skm_count   one thread per read: superkmers and packed bytes;
//   k_plain_skm_write   one thread per read: descriptors and packed bases;
//   then the same bin prefix / bin scatter as the fused path.
// Count (reference: kmc_counting_GPU per bin, kmer_counting.cu:59-199):
//   per bin: expand -> onesweep LSD radix sort -> run-length count.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "kernels.h"
#include "minimizer.cuh"
#include "onesweep.h"

using namespace gkc;

namespace gkc {

__global__ void k_plain_minimizer(const uint8_t *reads, const uint64_t *nbytes_dev, uint64_t nb_max,
                                  const uint32_t *rs_bits, int k, int p, int filter, uint32_t *mm) {
  const uint64_t nbytes = nbytes_dev ? *nbytes_dev : nb_max;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nbytes;
       s += (uint64_t)gridDim.x * blockDim.x) {
    if (!global_window_valid(rs_bits, nbytes, s, k)) continue;
    mm[s] = exact_window_minimizer([&](int i) { return global_code(reads, nbytes, (int64_t)s + i); }, k, p, filter);
  }
}

__global__ void k_plain_skm_count(const uint64_t *offs, uint64_t n_reads, const uint32_t *mm, int k,
                                  unsigned long long *nskm, unsigned long long *nbytes) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n_reads;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = offs[r], len = offs[r + 1] - b;
    unsigned long long cs = 0, cb = 0;
    if (len >= (uint64_t)k) {
      const uint64_t W = len - k + 1;
      uint64_t s0 = 0;
      for (uint64_t i = 1; i <= W; i++) {
        if (i == W || mm[b + i] != mm[b + i - 1]) {
          cs++;
          cb += (i - s0 + k - 1 + 3) / 4;
          s0 = i;
        }
      }
    }
    nskm[r] = cs;
    nbytes[r] = cb;
  }
}

__global__ void k_plain_skm_write(const uint8_t *reads, const uint64_t *offs, uint64_t n_reads,
                                  const uint32_t *mm, int k, uint32_t nbins, const uint64_t *skm_off,
                                  const uint64_t *byte_off, uint64_t *desc, uint32_t *skm_mm,
                                  uint8_t *packed, unsigned long long *bin_nskm,
                                  unsigned long long *bin_nkmers, uint32_t *err) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n_reads;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = offs[r], len = offs[r + 1] - b;
    if (len < (uint64_t)k) continue;
    const uint64_t W = len - k + 1;
    uint64_t si = skm_off[r], bo = byte_off[r], s0 = 0;
    for (uint64_t i = 1; i <= W; i++) {
      if (i == W || mm[b + i] != mm[b + i - 1]) {
        const uint64_t L = i - s0 + k - 1;
        if (L > 0xFFFFFFu) atomicOr(err, ERR_BAD_READ);
        desc[si] = (bo << 24) | (L & 0xFFFFFFu);
        const uint32_t m = mm[b + s0];
        skm_mm[si] = m;
        atomicAdd(&bin_nskm[m % nbins], 1ull);
        atomicAdd(&bin_nkmers[m % nbins], (unsigned long long)(i - s0));
        for (uint64_t q = 0; q < (L + 3) / 4; q++) {
          uint32_t byte = 0;
          for (int t = 0; t < 4; t++) {
            uint64_t j = 4 * q + t;
            uint32_t c = j < L ? (code_of_byte(reads[b + s0 + j]) & 3u) : 0u;
            byte = (byte << 2) | c;
          }
          packed[bo + q] = (uint8_t)byte;
        }
        bo += (L + 3) / 4;
        si++;
        s0 = i;
      }
    }
  }
}

// ---- per-bin counting ----

template <typename K>
__global__ void k_plain_expand(const uint64_t *desc, const uint8_t *packed, uint64_t s0, uint64_t s1,
                               const uint64_t *kmer_off, uint64_t k0, int k, K *keys) {
  for (uint64_t i = s0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < s1;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t d = desc[i];
    const uint64_t off = d >> 24;
    const uint32_t len = (uint32_t)(d & 0xFFFFFFu);
    if (len < (uint32_t)k) continue;
    const K mask = kmer_mask<K>(k);
    K x = 0;
    uint64_t w = kmer_off[i] - k0;
    for (uint32_t j = 0; j < len; j++) {
      uint32_t c = (packed[off + j / 4] >> (6 - 2 * (j & 3u))) & 3u;
      x = ((x << 2) | (K)c) & mask;
      if (j + 1 >= (uint32_t)k) {
        K rc = revcomp_k<K>(x, k);  // reference canonicalkmer, kmer_counting.cu:33-44
        keys[w++] = x < rc ? x : rc;
      }
    }
  }
}

__global__ void k_plain_nk(const uint64_t *desc, const unsigned long long *n_skm, int k,
                           unsigned long long *nk) {
  const uint64_t n = *n_skm;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t len = (uint32_t)(desc[i] & 0xFFFFFFu);
    nk[i] = len >= (uint32_t)k ? len - k + 1 : 0;
  }
}

constexpr int RLE_NT = 256;
constexpr int RLE_ITEMS = 8;
constexpr int RLE_TILE = RLE_NT * RLE_ITEMS;

template <typename K>
__global__ void k_rle_mark(const K *a, uint64_t n, unsigned long long *blk) {
  __shared__ uint64_t tmp[32];
  uint64_t base = (uint64_t)blockIdx.x * RLE_TILE + (uint64_t)threadIdx.x * RLE_ITEMS;
  uint64_t c = 0;
  for (int t = 0; t < RLE_ITEMS; t++) {
    uint64_t i = base + t;
    if (i < n) c += (i == 0 || a[i] != a[i - 1]);
  }
  c = block_sum_u64<RLE_NT>(c, tmp);
  if (threadIdx.x == 0) blk[blockIdx.x] = c;
}

template <typename K>
__global__ void k_rle_emit(const K *a, uint64_t n, const uint64_t *blk_off,
                           const unsigned long long *out_cursor, K *out_keys, uint64_t *starts) {
  __shared__ uint32_t tmp[64];
  uint64_t base = (uint64_t)blockIdx.x * RLE_TILE + (uint64_t)threadIdx.x * RLE_ITEMS;
  uint32_t c = 0;
  for (int t = 0; t < RLE_ITEMS; t++) {
    uint64_t i = base + t;
    if (i < n) c += (i == 0 || a[i] != a[i - 1]);
  }
  uint32_t total;
  uint64_t idx = blk_off[blockIdx.x] + block_exclusive_scan<RLE_NT>(c, tmp, &total);
  const uint64_t ob = *out_cursor;
  for (int t = 0; t < RLE_ITEMS; t++) {
    uint64_t i = base + t;
    if (i < n && (i == 0 || a[i] != a[i - 1])) {
      out_keys[ob + idx] = a[i];
      starts[idx] = i;
      idx++;
    }
  }
}

__global__ void k_rle_counts(const uint64_t *starts, const uint64_t *blk_off, uint64_t n_blk,
                             uint64_t n, const unsigned long long *out_cursor, uint32_t *counts) {
  const uint64_t D = blk_off[n_blk];
  const uint64_t ob = *out_cursor;
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < D;
       j += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t e = j + 1 < D ? starts[j + 1] : n;
    uint64_t run = e - starts[j];
    counts[ob + j] = run > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)run;
  }
}

__global__ void k_rle_advance(const uint64_t *blk_off, uint64_t n_blk, unsigned long long *out_cursor,
                              uint64_t *bin_out, uint32_t b, int empty) {
  bin_out[b] = *out_cursor;
  if (!empty) *out_cursor += blk_off[n_blk];
  bin_out[b + 1] = *out_cursor;
}

// Distinct keys of sorted[0, n) to out_keys (after *cursor) and the index of
// each one's first occurrence to starts: the run-length kernels above.
uint64_t rle_block_count(uint64_t n) { return (n + RLE_TILE - 1) / RLE_TILE; }

template <typename K>
void rle_runs(const K *sorted, uint64_t n, unsigned long long *blk, uint64_t *blk_off, uint64_t *tmp,
              const unsigned long long *cursor, K *out_keys, uint64_t *starts, cudaStream_t st) {
  const uint64_t nblk = rle_block_count(n);
  if (nblk == 0) return;
  k_rle_mark<K><<<(unsigned)nblk, RLE_NT, 0, st>>>(sorted, n, blk);
  scan_u64(blk, blk_off, nblk, tmp, st);
  k_rle_emit<K><<<(unsigned)nblk, RLE_NT, 0, st>>>(sorted, n, blk_off, cursor, out_keys, starts);
}
template void rle_runs<uint64_t>(const uint64_t *, uint64_t, unsigned long long *, uint64_t *, uint64_t *,
                                 const unsigned long long *, uint64_t *, uint64_t *, cudaStream_t);
template void rle_runs<u128>(const u128 *, uint64_t, unsigned long long *, uint64_t *, uint64_t *,
                             const unsigned long long *, u128 *, uint64_t *, cudaStream_t);

}  // namespace gkc

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

gkc_status partition_plain_impl(gkc_ctx *c, const gkc_params *prm, const char *d_reads,
                                uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads) {
  const uint32_t nbins = (uint32_t)prm->nbins;
  const uint8_t *src = reinterpret_cast<const uint8_t *>(d_reads);
  const uint64_t *offs = d_offs;
  const uint64_t *nbytes_dev = nullptr;
  WS(cur, unsigned long long, "cursors", 4);
  WS(err, uint32_t, "err", 4);
  CK(cudaMemsetAsync(cur, 0, 32, c->st));
  CK(cudaMemsetAsync(err, 0, 16, c->st));
  const unsigned grid = c->n_sms * 8;
  c->part_hpc_reads = nullptr;
  c->part_hpc_offs = nullptr;
  c->part_hpc_orig = nullptr;
  if (prm->hpc) {
    WS(runlen, unsigned long long, "hpc_runlen", n_reads + 1);
    WS(hoffs, uint64_t, "hpc_offs", n_reads + 2);
    WS(hreads, uint8_t, "hpc_reads", n_bytes + 64);
    WS(horig, int32_t, "hpc_orig", n_bytes + 16);
    WS(stmp, uint64_t, "scan_tmp", scan_u64_tmp_words(n_reads + 1) + 8);
    k_hpc_count<<<grid, 256, 0, c->st>>>(src, offs, n_reads, runlen);
    scan_u64(runlen, hoffs, n_reads, stmp, c->st);
    k_hpc_write<<<grid, 256, 0, c->st>>>(src, offs, n_reads, hoffs, hreads, horig);
    c->launches += 6;
    src = hreads;
    offs = hoffs;
    nbytes_dev = hoffs + n_reads;
    c->part_hpc_reads = (const char *)hreads;
    c->part_hpc_offs = hoffs;
    c->part_hpc_orig = horig;
  }
  const uint64_t rs_words = (n_bytes + 1 + 31) / 32 + 2;
  WS(rs, uint32_t, "rs_bits", rs_words);
  CK(cudaMemsetAsync(rs, 0, rs_words * 4, c->st));
  k_read_start_bits<<<(unsigned)std::min<uint64_t>((n_reads + 256) / 256, 65535), 256, 0, c->st>>>(offs, n_reads, rs);
  WS(mm, uint32_t, "plain_mm", n_bytes + 1);
  k_plain_minimizer<<<grid, 256, 0, c->st>>>(src, nbytes_dev, n_bytes, rs, prm->k, prm->p, c->filter, mm);
  WS(nskm, unsigned long long, "plain_nskm", n_reads + 1);
  WS(nbyt, unsigned long long, "plain_nbytes", n_reads + 1);
  WS(skm_off, uint64_t, "plain_skm_off", n_reads + 2);
  WS(byte_off, uint64_t, "plain_byte_off", n_reads + 2);
  WS(stmp2, uint64_t, "scan_tmp2", scan_u64_tmp_words(n_reads + 1) + 8);
  k_plain_skm_count<<<grid, 256, 0, c->st>>>(offs, n_reads, mm, prm->k, nskm, nbyt);
  scan_u64(nskm, skm_off, n_reads, stmp2, c->st);
  scan_u64(nbyt, byte_off, n_reads, stmp2, c->st);
  c->launches += 12;
  // sizes are needed on the host to allocate: this form synchronises here
  uint64_t tot[2];
  CK(cudaMemcpyAsync(&tot[0], skm_off + n_reads, 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(&tot[1], byte_off + n_reads, 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const uint64_t n_skm = tot[0], n_packed = tot[1];
  WS(desc, uint64_t, "skm_desc_tile", n_skm + 1);
  WS(smm, uint32_t, "skm_mm_tile", n_skm + 1);
  WS(packed, uint8_t, "packed", n_packed + 16);
  WS(bin_nskm, unsigned long long, "bin_nskm", nbins + 1);
  WS(bin_nkm, unsigned long long, "bin_nkmers", nbins + 1);
  CK(cudaMemsetAsync(bin_nskm, 0, (nbins + 1) * 8, c->st));
  CK(cudaMemsetAsync(bin_nkm, 0, (nbins + 1) * 8, c->st));
  k_plain_skm_write<<<grid, 256, 0, c->st>>>(src, offs, n_reads, mm, prm->k, nbins, skm_off, byte_off,
                                             desc, smm, packed, bin_nskm, bin_nkm, err);
  unsigned long long hc[2] = {n_skm, n_packed};
  CK(cudaMemcpyAsync(cur, hc, 16, cudaMemcpyHostToDevice, c->st));
  WS(bin_start, uint64_t, "bin_start", nbins + 1);
  WS(bin_kstart, uint64_t, "bin_kstart", nbins + 1);
  k_bin_prefix<<<1, 32, 0, c->st>>>(bin_nskm, bin_nkm, nbins, bin_start, bin_kstart);
  WS(bfill, unsigned long long, "bin_fill", nbins + 1);
  CK(cudaMemsetAsync(bfill, 0, (nbins + 1) * 8, c->st));
  WS(bdesc, uint64_t, "skm_desc_bin", n_skm + 1);
  WS(bmm, uint32_t, "skm_mm_bin", n_skm + 1);
  k_bin_scatter<<<grid, 256, 0, c->st>>>(cur, desc, smm, nbins, bin_start, bfill, bdesc, bmm,
                                         nullptr, nullptr, err);
  c->launches += 4;
  CK(cudaPeekAtLastError());
  c->part_cap_skm = n_skm + 1;
  c->part_cap_bytes = n_packed + 16;
  c->part_nbytes_dev = nbytes_dev;
  // totals for the view
  DevTotals *h = c->h_tot;
  std::memset(h, 0, sizeof(*h));
  uint64_t nkm = 0, nbh = n_bytes;
  CK(cudaMemcpyAsync(&nkm, bin_kstart + nbins, 8, cudaMemcpyDeviceToHost, c->st));
  if (nbytes_dev) CK(cudaMemcpyAsync(&nbh, nbytes_dev, 8, cudaMemcpyDeviceToHost, c->st));
  uint32_t e = 0;
  CK(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (e & ERR_BAD_READ) return ctx_fail(c, GKC_ERR_INVALID_ARG, "read longer than supported");
  gkc_partition_view &v = c->pv;
  memset(&v, 0, sizeof(v));
  v.n_reads = n_reads;
  v.n_bases = nbh;
  v.n_superkmers = n_skm;
  v.n_packed_bytes = n_packed;
  v.n_kmers = nkm;
  v.nbins = nbins;
  v.bin_skm_off = bin_start;
  v.bin_kmer_off = bin_kstart;
  v.skm_desc = bdesc;
  v.skm_minimizer = bmm;
  v.packed = packed;
  c->part_packed = packed;
  v.hpc_reads = c->part_hpc_reads;
  v.hpc_offs = c->part_hpc_offs;
  v.hpc_orig_pos = c->part_hpc_orig;
  c->pp = *prm;
  c->have_part = true;
  return GKC_OK;
}

template <typename K>
static gkc_status count_plain_t(gkc_ctx *c, const gkc_params *prm) {
  const uint32_t nbins = c->pv.nbins;
  const int k = prm->k;
  const uint64_t n_skm = c->pv.n_superkmers, N = c->pv.n_kmers;
  std::vector<uint64_t> bs(nbins + 1), bk(nbins + 1);
  CK(cudaMemcpyAsync(bs.data(), c->pv.bin_skm_off, (nbins + 1) * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(bk.data(), c->pv.bin_kmer_off, (nbins + 1) * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  WS(nk, unsigned long long, "plain_nk", n_skm + 1);
  WS(kmer_off, uint64_t, "plain_kmer_off", n_skm + 2);
  WS(stmp, uint64_t, "scan_tmp2", scan_u64_tmp_words(n_skm + 1) + 8);
  WS(ncount, unsigned long long, "plain_nskm_dev", 2);
  unsigned long long hn = n_skm;
  CK(cudaMemcpyAsync(ncount, &hn, 8, cudaMemcpyHostToDevice, c->st));
  const unsigned grid = c->n_sms * 8;
  k_plain_nk<<<grid, 256, 0, c->st>>>(c->pv.skm_desc, ncount, k, nk);
  scan_u64(nk, kmer_off, n_skm, stmp, c->st);
  c->launches += 5;
  WS(keys, K, "keys", N + 16);
  WS(alt, K, "keys_alt", N + 16);
  WS(counts, uint32_t, "counts", N + 16);
  WS(out_keys, K, "plain_out_keys", N + 16);
  WS(bin_n, uint64_t, "plain_bin_n", nbins + 1);
  std::vector<uint64_t> hbn(nbins + 1);
  for (uint32_t b = 0; b < nbins; b++) hbn[b] = bk[b + 1] - bk[b];
  CK(cudaMemcpyAsync(bin_n, hbn.data(), (nbins + 1) * 8, cudaMemcpyHostToDevice, c->st));
  uint64_t max_bin = 0;
  for (uint32_t b = 0; b < nbins; b++) max_bin = std::max(max_bin, hbn[b]);
  WS(os_hist, unsigned long long, "os_hist", 16 * 256);
  WS(os_lb, unsigned long long, "os_lookback", onesweep_lookback_words(max_bin + 1));
  WS(os_ticket, unsigned long long, "os_ticket", 2);
  WS(err, uint32_t, "err", 4);
  const uint64_t rle_blocks = (max_bin + RLE_TILE - 1) / RLE_TILE + 1;
  WS(rle_blk, unsigned long long, "rle_blk", rle_blocks + 1);
  WS(rle_off, uint64_t, "rle_off", rle_blocks + 2);
  WS(rle_tmp, uint64_t, "rle_tmp", scan_u64_tmp_words(rle_blocks) + 8);
  WS(starts, uint64_t, "rle_starts", max_bin + 1);
  WS(out_cursor, unsigned long long, "out_cursor", 2);
  WS(bin_out, uint64_t, "bin_out", nbins + 1);
  CK(cudaMemsetAsync(out_cursor, 0, 16, c->st));
  CK(cudaMemsetAsync(bin_out, 0, (nbins + 1) * 8, c->st));
  OnesweepScratch os{os_hist, os_lb, os_ticket, err, c->n_sms * 4};
  for (uint32_t b = 0; b < nbins; b++) {
    const uint64_t n = hbn[b];
    K *kb = keys + bk[b], *ab = alt + bk[b];
    if (n) {
      k_plain_expand<K><<<grid, 256, 0, c->st>>>(c->pv.skm_desc, c->pv.packed, bs[b], bs[b + 1],
                                                  kmer_off, bk[b], k, kb);
      c->launches++;
      OnesweepStatus r = onesweep_sort<K>(kb, ab, bin_n + b, n, 2 * k, os, c->st, &c->launches);
      const K *sorted = r.result_in_alt ? ab : kb;
      const uint64_t nblk = (n + RLE_TILE - 1) / RLE_TILE;
      k_rle_mark<K><<<(unsigned)nblk, RLE_NT, 0, c->st>>>(sorted, n, rle_blk);
      scan_u64(rle_blk, rle_off, nblk, rle_tmp, c->st);
      k_rle_emit<K><<<(unsigned)nblk, RLE_NT, 0, c->st>>>(sorted, n, rle_off, out_cursor, out_keys, starts);
      k_rle_counts<<<grid, 256, 0, c->st>>>(starts, rle_off, nblk, n, out_cursor, counts);
      k_rle_advance<<<1, 1, 0, c->st>>>(rle_off, nblk, out_cursor, bin_out, b, 0);
      c->launches += 8;
    } else {
      k_rle_advance<<<1, 1, 0, c->st>>>(rle_off, 0, out_cursor, bin_out, b, 1);
      c->launches++;
    }
    CK(cudaPeekAtLastError());
  }
  uint64_t nd = 0;
  uint32_t e = 0;
  CK(cudaMemcpyAsync(&nd, out_cursor, 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (e & ERR_SPIN_TIMEOUT) return ctx_fail(c, GKC_ERR_DEVICE_TIMEOUT, "onesweep look-back timed out");
  gkc_count_view &v = c->cv;
  memset(&v, 0, sizeof(v));
  v.n_distinct = nd;
  v.n_kmers = N;
  v.nbins = nbins;
  v.key_words = k <= 32 ? 1 : 2;
  v.bin_off = bin_out;
  v.keys = reinterpret_cast<const uint64_t *>(out_keys);
  v.counts = counts;
  c->ck = k;
  c->have_count = true;
  c->count_gen++;
  return GKC_OK;
}

gkc_status count_plain_impl(gkc_ctx *c, const gkc_params *prm) {
  if (!c->have_part) return ctx_fail(c, GKC_ERR_INVALID_ARG, "no partition in the context");
  CK(cudaMemsetAsync(c->bufs["err"].p, 0, 16, c->st));
  if (prm->k <= 32) return count_plain_t<uint64_t>(c, prm);
  return count_plain_t<u128>(c, prm);
}

// ---------------------------------------------------------------------------
// Counting one group of packed superkmers without allocating any memory.
//
// Some callers cannot allocate device memory while they run: a host program
// that hands the GPU to this library inside its own fixed memory pool, a
// framework whose allocator owns all of HBM, or code on a path where a
// cudaMalloc would synchronise the device or fail under a hard memory cap.
// This entry point serves them.  It runs the same kernels as the per-stage
// counting path above (expand, onesweep radix sort, run-length encoding), but
// all its scratch memory is carved out of one fixed array of device memory
// that the library declares at file scope; the caller passes only the inputs
// and the output buffers.  Every GPU that loads the library holds the array
// (about 23 MB) until the process exits.
// ---------------------------------------------------------------------------
namespace gkc {
namespace noalloc {

constexpr uint64_t kMaxKmers = 1ull << 20;  // k-mers per call
constexpr uint64_t kMaxSkm = 1ull << 17;    // superkmers per call
constexpr int kMaxDevices = 64;

constexpr uint64_t round_up(uint64_t w) { return (w + 31) & ~31ull; }  // 256-byte steps
constexpr uint64_t kOsTileMax = 4096;  // keys per onesweep tile (checked at set-up)
constexpr uint64_t kRleBlocks = (kMaxKmers + RLE_TILE - 1) / RLE_TILE + 1;
// word offsets of the parts of the array
constexpr uint64_t W_SORT = 0;
constexpr uint64_t W_STARTS = W_SORT + round_up(kMaxKmers + 16);
constexpr uint64_t W_NBYTES = W_STARTS + round_up(kMaxKmers + 16);
constexpr uint64_t W_BOFF = W_NBYTES + round_up(kMaxSkm + 2);
constexpr uint64_t W_NK = W_BOFF + round_up(kMaxSkm + 2);
constexpr uint64_t W_KOFF = W_NK + round_up(kMaxSkm + 2);
constexpr uint64_t W_DESC = W_KOFF + round_up(kMaxSkm + 2);
constexpr uint64_t W_STMP = W_DESC + round_up(kMaxSkm + 2);
constexpr uint64_t W_HIST = W_STMP + round_up(kMaxSkm / 1024 + 16);
constexpr uint64_t W_LB = W_HIST + round_up(16 * 256);
constexpr uint64_t W_TICKET = W_LB + round_up(((kMaxKmers + kOsTileMax - 1) / kOsTileMax + 1) * 256);
constexpr uint64_t W_ERR = W_TICKET + 32;
constexpr uint64_t W_RBLK = W_ERR + 32;
constexpr uint64_t W_ROFF = W_RBLK + round_up(kRleBlocks + 1);
constexpr uint64_t W_RTMP = W_ROFF + round_up(kRleBlocks + 2);
constexpr uint64_t W_CURSOR = W_RTMP + round_up(kRleBlocks / 1024 + 16);
constexpr uint64_t W_BINOUT = W_CURSOR + 32;
constexpr uint64_t kWords = W_BINOUT + 32;

// The scratch array.  In host code this name is only a stand-in for the
// device symbol, not a device address; the host takes the real address with
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned long long scratch[kWords];

// per superkmer: packed bytes, k-mers; flags lengths the descriptor cannot hold
__global__ void k_prepare(const uint32_t *len, uint64_t n, int k, unsigned long long *nbytes,
                          unsigned long long *nk, uint32_t *err) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t l = len[i];
    if (l > 0xFFFFFFu) atomicOr(err, ERR_BAD_READ);
    nbytes[i] = (l + 3u) / 4u;
    nk[i] = l >= (uint32_t)k ? l - k + 1 : 0;
  }
}

// descriptor of superkmer i: (first packed byte << 24) | length
__global__ void k_desc(const uint32_t *len, const uint64_t *boff, uint64_t n, uint64_t *desc) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    desc[i] = (boff[i] << 24) | (len[i] & 0xFFFFFFu);
}

struct Dev {
  unsigned long long *base = nullptr;
  int sms = 0;
};
static std::mutex g_mu;
static Dev g_dev[kMaxDevices];

// Set-up for the current device, once: the array's device address and the
// SM count.  With lazy module loading (the CUDA default) the library's
// kernels and the array itself are loaded onto the device by this first
// lookup, so the first call does take device memory for them.  The address is
// kept for the life of the process: after cudaDeviceReset it would be stale.
static gkc_status setup(int dev, Dev *out) {
  if (dev < 0 || dev >= kMaxDevices) return GKC_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_dev[dev].base) {
    if (onesweep_lookback_words(kMaxKmers) > W_TICKET - W_LB) return GKC_ERR_INTERNAL;
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return GKC_ERR_CUDA;
    }
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || sms <= 0) {
      cudaGetLastError();
      return GKC_ERR_CUDA;
    }
    g_dev[dev].base = static_cast<unsigned long long *>(p);
    g_dev[dev].sms = sms;
  }
  *out = g_dev[dev];
  return GKC_OK;
}

}  // namespace noalloc
}  // namespace gkc

#define NA_CK(call)                    \
  do {                                 \
    if ((call) != cudaSuccess) {       \
      cudaGetLastError();              \
      return GKC_ERR_CUDA;             \
    }                                  \
  } while (0)

extern "C" gkc_status gkc_count_superkmers_device_noalloc(int k, const uint32_t *d_skm_len,
                                                          const uint8_t *d_packed, uint64_t n_skm,
                                                          uint64_t out_capacity, uint64_t *d_keys_out,
                                                          uint32_t *d_counts_out, uint64_t *n_distinct,
                                                          void *cuda_stream) {
  using namespace gkc;
  using namespace gkc::noalloc;
  if (k < 1 || k > 32 || !n_distinct) return GKC_ERR_INVALID_ARG;
  if (n_skm > kMaxSkm) return GKC_ERR_CAPACITY;
  if (n_skm && (!d_skm_len || !d_packed)) return GKC_ERR_INVALID_ARG;
  if (out_capacity && (!d_keys_out || !d_counts_out)) return GKC_ERR_INVALID_ARG;
  *n_distinct = 0;
  if (n_skm == 0) return GKC_OK;
  int dev = 0;
  NA_CK(cudaGetDevice(&dev));
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  // the call waits on its stream twice (to read the sizes, then the result):
  // on a stream that is being captured that would end the caller's capture,
  // so such a call is refused before any work is queued
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  NA_CK(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) return GKC_ERR_INVALID_ARG;
  Dev d;
  gkc_status s = setup(dev, &d);
  if (s != GKC_OK) return s;
  unsigned long long *w = d.base;
  auto u64p = [&](uint64_t off) { return reinterpret_cast<uint64_t *>(w + off); };
  uint32_t *err = reinterpret_cast<uint32_t *>(w + W_ERR);
  const unsigned grid = (unsigned)d.sms * 8;

  // the array keeps the previous call's contents: clear what must start at zero
  NA_CK(cudaMemsetAsync(w + W_ERR, 0, 32 * 8, st));
  NA_CK(cudaMemsetAsync(w + W_CURSOR, 0, 32 * 8, st));
  NA_CK(cudaMemsetAsync(w + W_BINOUT, 0, 32 * 8, st));
  k_prepare<<<grid, 256, 0, st>>>(d_skm_len, n_skm, k, w + W_NBYTES, w + W_NK, err);
  scan_u64(w + W_NBYTES, u64p(W_BOFF), n_skm, u64p(W_STMP), st);
  scan_u64(w + W_NK, u64p(W_KOFF), n_skm, u64p(W_STMP), st);
  NA_CK(cudaPeekAtLastError());
  uint64_t total = 0;
  uint32_t e = 0;
  NA_CK(cudaMemcpyAsync(&total, u64p(W_KOFF) + n_skm, 8, cudaMemcpyDeviceToHost, st));
  NA_CK(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
  if (e & ERR_BAD_READ) return GKC_ERR_INVALID_ARG;  // a length above 2^24 - 1
  if (total > kMaxKmers || total > out_capacity) return GKC_ERR_CAPACITY;
  if (total == 0) return GKC_OK;

  k_desc<<<grid, 256, 0, st>>>(d_skm_len, u64p(W_BOFF), n_skm, u64p(W_DESC));
  uint64_t *keys = u64p(W_SORT);
  k_plain_expand<uint64_t><<<grid, 256, 0, st>>>(u64p(W_DESC), d_packed, 0, n_skm, u64p(W_KOFF), 0, k,
                                                  keys);
  // the caller's key buffer serves as the sort's second buffer
  OnesweepScratch os{w + W_HIST, w + W_LB, w + W_TICKET, err, d.sms * 4};
  uint32_t launches = 0;
  OnesweepStatus r = onesweep_sort<uint64_t>(keys, d_keys_out, u64p(W_KOFF) + n_skm, total, 2 * k, os,
                                             st, &launches);
  if (r.result_in_alt) NA_CK(cudaMemcpyAsync(keys, d_keys_out, total * 8, cudaMemcpyDeviceToDevice, st));
  const uint64_t nblk = (total + RLE_TILE - 1) / RLE_TILE;
  unsigned long long *cursor = w + W_CURSOR;
  k_rle_mark<uint64_t><<<(unsigned)nblk, RLE_NT, 0, st>>>(keys, total, w + W_RBLK);
  scan_u64(w + W_RBLK, u64p(W_ROFF), nblk, u64p(W_RTMP), st);
  k_rle_emit<uint64_t><<<(unsigned)nblk, RLE_NT, 0, st>>>(keys, total, u64p(W_ROFF), cursor, d_keys_out,
                                                          u64p(W_STARTS));
  k_rle_counts<<<grid, 256, 0, st>>>(u64p(W_STARTS), u64p(W_ROFF), nblk, total, cursor, d_counts_out);
  k_rle_advance<<<1, 1, 0, st>>>(u64p(W_ROFF), nblk, cursor, u64p(W_BINOUT), 0, 0);
  NA_CK(cudaPeekAtLastError());
  uint64_t nd = 0;
  NA_CK(cudaMemcpyAsync(&nd, cursor, 8, cudaMemcpyDeviceToHost, st));
  NA_CK(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
  if (e & ERR_SPIN_TIMEOUT) return GKC_ERR_DEVICE_TIMEOUT;
  *n_distinct = nd;
  return GKC_OK;
}
