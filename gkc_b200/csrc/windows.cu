// Per-window outputs over the read CSR:
//  * gkc_minimizers_device: the canonical minimizer of every k-window with the
//    position of the selected p-mer inside the window and its strand.  The
//    reference declares these outputs (d_mm_pos / d_mm_strand,
//    gkc_cuda.cu:159-160; CountTask::StoreMinimizerPos, gkc_cuda.hpp:50) but
//    never fills them; the definition here is the rightmost p-mer whose
//    passing forward or reverse-complement value equals the window's
//    minimizer (the ">=" updates at gkc_cuda.cu:283-284 let later candidates
//    win ties), strand -1 for a palindromic p-mer, 1 for the reverse
//    complement, 0 forward.
//  * gkc_subsample_positions_device: the canonical k-mers whose window
//    minimizer % mod == 0, each with the ascending list of its window starts
//    (README.md:16 use case; no reference code).
// Windows are indexed by their first byte's position in d_reads; a window
// that does not lie inside one read is invalid.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "ctx.h"
#include "kernels.h"
#include "minimizer.cuh"
#include "onesweep.h"

namespace gkc {

// Bit i set for every read start offs[r] (r <= n_reads, so the end of the
// last read is marked too).  Offsets past n_bytes are flagged, not written.
__global__ void k_window_starts(const uint64_t *offs, uint64_t n_reads, uint64_t n_bytes,
                                uint32_t *bits, uint32_t *err) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r <= n_reads;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t pos = offs[r];
    if (pos > n_bytes || (r > 0 && offs[r - 1] > pos)) {
      atomicOr(err, ERR_BAD_READ);
      continue;
    }
    atomicOr(&bits[pos >> 5], 1u << (pos & 31));
  }
}

// Window [i, i + k) inside one read: lo <= i, i + k <= hi, and no read start
// at positions i+1 .. i+k-1.
GKC_DEV bool window_inside(const uint32_t *bits, uint64_t i, int k, uint64_t lo, uint64_t hi) {
  if (i < lo || i + k > hi) return false;
  for (uint64_t q = i + 1; q < i + k;) {
    const uint32_t w = bits[q >> 5] >> (q & 31);
    const uint64_t left = i + k - q, room = 32 - (q & 31);
    const uint32_t span = (uint32_t)(left < room ? left : room);
    const uint32_t m = span == 32 ? 0xFFFFFFFFu : ((1u << span) - 1u);
    if (w & m) return false;
    q += span;
  }
  return true;
}

struct WinMin {
  uint32_t mm;
  uint8_t pos;
  int8_t strand;
};

// Minimizer, position and strand of the window at i (inside a read).
GKC_DEV WinMin window_min_pos(const uint8_t *reads, uint64_t i, int k, int p, int filter) {
  WinMin w;
  w.mm = exact_window_minimizer([&](int j) { return code_of_byte(reads[i + j]); }, k, p, filter);
  const uint32_t M = 0xFFFFFFFFu >> (32 - 2 * p);
  uint32_t f = 0, r = 0;
  int bpos = 255, bstr = 0;
  for (int j = 0; j < k; j++) {
    const uint32_t c0 = code_of_byte(reads[i + j]);
    const uint32_t c = c0 & 3u;                          // N counts as T here
    const uint32_t cc = (c0 == 255u ? 255u : 3u - c0) & 3u;  // and its complement as T
    f = ((f << 2) | c) & M;
    r = (r >> 2) | (cc << (2 * p - 2));
    if (j + 1 >= p) {
      const bool mf = mm_filter(f, p, filter) && f == w.mm;
      const bool mr = mm_filter(r, p, filter) && r == w.mm;
      if (mf || mr) {
        bpos = j + 1 - p;
        bstr = (f == r) ? -1 : (mr ? 1 : 0);
      }
    }
  }
  w.pos = (uint8_t)bpos;
  w.strand = (int8_t)bstr;
  return w;
}

__global__ void k_window_minimizers(const uint8_t *reads, uint64_t n_bytes, const uint64_t *offs,
                                    uint64_t n_reads, const uint32_t *bits, int k, int p, int filter,
                                    uint32_t *mm, uint8_t *pos, int8_t *strand) {
  const uint64_t lo = offs[0], hi = offs[n_reads];
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_bytes;
       i += (uint64_t)gridDim.x * blockDim.x) {
    WinMin w{0xFFFFFFFFu, 255, 0};
    if (hi <= n_bytes && window_inside(bits, i, k, lo, hi)) w = window_min_pos(reads, i, k, p, filter);
    mm[i] = w.mm;
    if (pos) pos[i] = w.pos;
    if (strand) strand[i] = w.strand;
  }
}

// ---- subsampling: windows whose minimizer % mod == 0, in window order ----

constexpr int SUB_NT = 256;
constexpr int SUB_ITEMS = 16;
constexpr int SUB_TILE = SUB_NT * SUB_ITEMS;  // windows per tile = 128 bitmap words

// Tile t covers windows [t*SUB_TILE, (t+1)*SUB_TILE): selection bitmap and count.
__global__ void k_sub_flags(const uint8_t *reads, uint64_t n_bytes, const uint64_t *offs,
                            uint64_t n_reads, const uint32_t *bits, int k, int p, int filter,
                            uint32_t mod, uint32_t *sel, unsigned long long *tile_cnt) {
  __shared__ uint64_t tmp[32];
  const uint64_t lo = offs[0], hi = offs[n_reads];
  const uint64_t t = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t cnt = 0;
  // warp w handles bitmap words t*128 + w*16 + r: 32 consecutive windows each
  for (int r = 0; r < SUB_ITEMS; r++) {
    const uint64_t word = t * (SUB_TILE / 32) + (uint64_t)warp * SUB_ITEMS + r;
    const uint64_t i = word * 32 + lane;
    bool f = false;
    if (i < n_bytes && hi <= n_bytes && window_inside(bits, i, k, lo, hi)) {
      const uint32_t m = exact_window_minimizer([&](int j) { return code_of_byte(reads[i + j]); }, k, p, filter);
      f = (m % mod) == 0u;
    }
    const uint32_t b = __ballot_sync(0xffffffffu, f);
    if (lane == 0 && word * 32 < n_bytes) sel[word] = b;
    cnt += __popc(b) * (lane == 0);
  }
  cnt = block_sum_u64<SUB_NT>(cnt, tmp);
  if (threadIdx.x == 0) tile_cnt[t] = cnt;
}

template <typename K>
GKC_DEV K window_canonical(const uint8_t *reads, uint64_t i, int k) {
  K x = 0;
  for (int j = 0; j < k; j++) x = (x << 2) | (K)(code_of_byte(reads[i + j]) & 3u);  // N -> T
  const K r = revcomp_k<K>(x, k);
  return x < r ? x : r;
}

// Writes (canonical key, window start) of the selected windows in window order.
template <typename K>
__global__ void k_sub_write(const uint8_t *reads, uint64_t n_bytes, const uint32_t *sel,
                            const uint64_t *tile_off, int k, K *keys, uint32_t *posv) {
  __shared__ uint32_t tmp[64];
  const uint64_t t = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // thread (warp, lane) owns bitmap word t*128 + warp*16 + lane/2, half lane&1
  const uint64_t word = t * (SUB_TILE / 32) + (uint64_t)warp * SUB_ITEMS + (lane >> 1);
  const bool in = word * 32 < n_bytes;
  uint32_t b = in ? sel[word] : 0u;
  b = (lane & 1) ? (b >> 16) : (b & 0xFFFFu);
  const uint32_t c = __popc(b);
  uint32_t total;
  uint64_t o = tile_off[t] + block_exclusive_scan<SUB_NT>(c, tmp, &total);
  const uint64_t i0 = word * 32 + (lane & 1) * 16;
  while (b) {
    const int q = __ffs(b) - 1;
    b &= b - 1;
    const uint64_t i = i0 + q;
    keys[o] = window_canonical<K>(reads, i, k);
    posv[o] = (uint32_t)i;
    o++;
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

static gkc_status check_window_args(gkc_ctx *c, const gkc_params *prm, const char *d_reads,
                                    uint64_t n_bytes, const uint64_t *d_offs, int kmax) {
  if (!c || !prm) return GKC_ERR_INVALID_ARG;
  if (prm->k < 1 || prm->k > kmax || prm->p < 3 || prm->p > 16 || prm->p > prm->k)
    return ctx_fail(c, GKC_ERR_INVALID_ARG, "need 3 <= p <= min(k, 16)");
  if (prm->hpc) return ctx_fail(c, GKC_ERR_INVALID_ARG, "run gkc_hpc_device first; hpc must be 0 here");
  if (n_bytes >= (1ull << 32)) return ctx_fail(c, GKC_ERR_INVALID_ARG, "positions are 32-bit");
  if (n_bytes && (!d_reads || !d_offs)) return ctx_fail(c, GKC_ERR_INVALID_ARG, "null input");
  return GKC_OK;
}

static gkc_status mark_starts(gkc_ctx *c, const uint64_t *d_offs, uint64_t n_reads, uint64_t n_bytes,
                              uint32_t **bits_out, uint32_t **err_out) {
  const uint64_t words = (n_bytes + 1) / 32 + 3;
  WS(bits, uint32_t, "win_bits", words);
  WS(err, uint32_t, "win_err", 4);
  CK(cudaMemsetAsync(bits, 0, words * 4, c->st));
  CK(cudaMemsetAsync(err, 0, 16, c->st));
  k_window_starts<<<(unsigned)std::min<uint64_t>((n_reads + 256) / 256, 65535), 256, 0, c->st>>>(
      d_offs, n_reads, n_bytes, bits, err);
  CK(cudaPeekAtLastError());
  *bits_out = bits;
  *err_out = err;
  return GKC_OK;
}

static gkc_status read_err(gkc_ctx *c, const uint32_t *err) {
  uint32_t e = 0;
  CK(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (e & ERR_BAD_READ) return ctx_fail(c, GKC_ERR_INVALID_ARG, "read offsets decrease or pass n_bytes");
  if (e & ERR_SPIN_TIMEOUT) return ctx_fail(c, GKC_ERR_DEVICE_TIMEOUT, "sort look-back timed out");
  return GKC_OK;
}

gkc_status gkc_minimizers_device(gkc_ctx *c, const gkc_params *prm, const char *d_reads,
                                 uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads,
                                 uint32_t *d_minimizer, uint8_t *d_pos, int8_t *d_strand) {
  gkc_status s = check_window_args(c, prm, d_reads, n_bytes, d_offs, 64);
  if (s != GKC_OK) return s;
  if (n_bytes == 0) return GKC_OK;
  if (!d_minimizer) return ctx_fail(c, GKC_ERR_INVALID_ARG, "null minimizer output");
  cudaSetDevice(c->dev);
  uint32_t *bits, *err;
  s = mark_starts(c, d_offs, n_reads, n_bytes, &bits, &err);
  if (s != GKC_OK) return s;
  k_window_minimizers<<<c->n_sms * 16, 256, 0, c->st>>>(reinterpret_cast<const uint8_t *>(d_reads), n_bytes,
                                                         d_offs, n_reads, bits, prm->k, prm->p, c->filter, d_minimizer,
                                                         d_pos, d_strand);
  CK(cudaPeekAtLastError());
  return read_err(c, err);
}

template <typename K>
static gkc_status subsample_t(gkc_ctx *c, const gkc_params *prm, uint32_t mod, const uint8_t *reads,
                              uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads,
                              gkc_poslist_view *out) {
  uint32_t *bits, *err;
  gkc_status s = mark_starts(c, d_offs, n_reads, n_bytes, &bits, &err);
  if (s != GKC_OK) return s;
  const uint64_t tiles = (n_bytes + SUB_TILE - 1) / SUB_TILE;
  WS(sel, uint32_t, "win_sel", tiles * (SUB_TILE / 32) + 1);
  WS(tcnt, unsigned long long, "win_tile_cnt", tiles + 1);
  WS(toff, uint64_t, "win_tile_off", tiles + 2);
  WS(stmp, uint64_t, "win_scan_tmp", scan_u64_tmp_words(tiles + 1) + 8);
  k_sub_flags<<<(unsigned)tiles, SUB_NT, 0, c->st>>>(reads, n_bytes, d_offs, n_reads, bits, prm->k, prm->p,
                                                     c->filter, mod, sel, tcnt);
  scan_u64(tcnt, toff, tiles, stmp, c->st);
  CK(cudaPeekAtLastError());
  uint64_t n = 0;
  CK(cudaMemcpyAsync(&n, toff + tiles, 8, cudaMemcpyDeviceToHost, c->st));
  s = read_err(c, err);  // synchronises
  if (s != GKC_OK) return s;
  WS(keys, K, "win_keys", n + 16);
  WS(alt, K, "win_keys_alt", n + 16);
  WS(pos, uint32_t, "win_pos", n + 16);
  WS(palt, uint32_t, "win_pos_alt", n + 16);
  WS(out_keys, K, "win_out_keys", n + 16);
  WS(pos_off, uint64_t, "win_pos_off", n + 2);
  if (n) {
    k_sub_write<K><<<(unsigned)tiles, SUB_NT, 0, c->st>>>(reads, n_bytes, sel, toff, prm->k, keys, pos);
    CK(cudaPeekAtLastError());
    WS(os_hist, unsigned long long, "win_os_hist", 16 * 256);
    WS(os_lb, unsigned long long, "win_os_lookback", onesweep_lookback_words(n + 1));
    WS(os_ticket, unsigned long long, "win_os_ticket", 2);
    OnesweepScratch os{os_hist, os_lb, os_ticket, err, c->n_sms * 4};
    // the selected count, on the device, for the sort
    const uint64_t *n_dev = toff + tiles;
    uint32_t launches = 0;
    OnesweepStatus r = onesweep_sort_kv<K>(keys, alt, pos, palt, n_dev, n, 2 * prm->k, os, c->st, &launches);
    const K *sk = r.result_in_alt ? alt : keys;
    const uint32_t *sp = r.result_in_alt ? palt : pos;
    // distinct keys and their first indices (= the position-list offsets)
    const uint64_t nblk = rle_block_count(n);
    WS(rblk, unsigned long long, "win_rle_blk", nblk + 1);
    WS(roff, uint64_t, "win_rle_off", nblk + 2);
    WS(rtmp, uint64_t, "win_rle_tmp", scan_u64_tmp_words(nblk + 1) + 8);
    WS(cur, unsigned long long, "win_cursor", 2);
    CK(cudaMemsetAsync(cur, 0, 16, c->st));
    rle_runs<K>(sk, n, rblk, roff, rtmp, cur, out_keys, pos_off, c->st);
    CK(cudaPeekAtLastError());
    uint64_t nd = 0;
    CK(cudaMemcpyAsync(&nd, roff + nblk, 8, cudaMemcpyDeviceToHost, c->st));
    s = read_err(c, err);
    if (s != GKC_OK) return s;
    uint64_t nn = n;
    CK(cudaMemcpyAsync(pos_off + nd, &nn, 8, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    out->n_distinct = nd;
    out->positions = sp;
  } else {
    uint64_t zero = 0;
    CK(cudaMemcpyAsync(pos_off, &zero, 8, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    out->n_distinct = 0;
    out->positions = pos;
  }
  out->n_positions = n;
  out->key_words = sizeof(K) / 8;
  out->keys = reinterpret_cast<const uint64_t *>(out_keys);
  out->pos_off = pos_off;
  return GKC_OK;
}

gkc_status gkc_subsample_positions_device(gkc_ctx *c, const gkc_params *prm, uint32_t mod,
                                          const char *d_reads, uint64_t n_bytes,
                                          const uint64_t *d_offs, uint64_t n_reads,
                                          gkc_poslist_view *out) {
  gkc_status s = check_window_args(c, prm, d_reads, n_bytes, d_offs, 64);
  if (s != GKC_OK) return s;
  if (!out || mod == 0) return ctx_fail(c, GKC_ERR_INVALID_ARG, "need mod >= 1 and an output view");
  memset(out, 0, sizeof(*out));
  out->key_words = prm->k <= 32 ? 1 : 2;
  if (n_bytes == 0) return GKC_OK;
  cudaSetDevice(c->dev);
  const uint8_t *reads = reinterpret_cast<const uint8_t *>(d_reads);
  if (prm->k <= 32) return subsample_t<uint64_t>(c, prm, mod, reads, n_bytes, d_offs, n_reads, out);
  return subsample_t<u128>(c, prm, mod, reads, n_bytes, d_offs, n_reads, out);
}
